// Per-instance vector reductions (mean projection, RMS), the CSR export of stencil
// matrices, grid metrics, and the C ABI housekeeping.
#include <string>
#include <cmath>
#include "phb_device.cuh"
#include "phb_launch.cuh"

namespace phb {

static thread_local std::string tlError;
void setErrorText(const char *msg) { tlError = msg ? msg : ""; }

constexpr int NW = PHB_TILE / 32;

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
	return v;
}

// Sums over each instance of comps components (POW 1: values, 2: squares). Partials per
// tile, reduced per instance by the last CTA in a fixed order. scratch layout (doubles):
// [0] ticket counter (must start at 0, is reset to 0), [8, 8+ninst*comps) results,
// then ntiles*comps partials.
template <typename S, int D, int POW>
__global__ void __launch_bounds__(PHB_TILE) kInstanceSums(Dom<S, D> dom, const S *__restrict__ x, int comps, double *scratch, int mode) {
	__shared__ int32_t sB[PHB_BREC];
	__shared__ double sm[3][NW];
	__shared__ bool isLast;
	int l0_, nc_;
	loadTile<S, D>(dom, sB, l0_, nc_);
	double v[3] = {0, 0, 0};
	for (int j_ = 0; j_ < CPT; ++j_) {
		Cell c;
		if (!cellAt<D>(sB, l0_, nc_, j_, c)) break;
		for (int k = 0; k < comps; ++k) {
			const double a = double(x[c.g + (int64_t)(comps - 1) * c.B[B_INSTOFF] + (int64_t)k * c.B[B_INSTN]]);
			v[k] += POW == 2 ? a * a : a;
		}
	}
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	for (int k = 0; k < comps; ++k) {
		const double s = wsum(v[k]);
		if (lane == 0) sm[k][warp] = s;
	}
	__syncthreads();
	double *res = scratch + 8;
	double *partial = res + dom.ninst * comps;
	unsigned int *counter = reinterpret_cast<unsigned int *>(scratch);
	if (threadIdx.x < comps) {
		double s = 0;
		for (int w = 0; w < NW; ++w) s += sm[threadIdx.x][w];
		partial[(size_t)blockIdx.x * comps + threadIdx.x] = s;
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		__threadfence();
		isLast = atomicAdd(counter, 1u) == gridDim.x - 1;
	}
	__syncthreads();
	if (!isLast) return;
	__threadfence();
	const int nsys = dom.ninst * comps;
	for (int s = warp; s < nsys; s += NW) {
		const int inst = s / comps, k = s - inst * comps;
		const int t0 = dom.insts[inst * PHB_IREC + I_TILESTART], tc = dom.insts[inst * PHB_IREC + I_TILECOUNT];
		double a = 0;
		for (int t = lane; t < tc; t += 32) a += __ldcg(partial + (size_t)(t0 + t) * comps + k);
		a = wsum(a);
		if (lane == 0) {
			const double n = double(dom.insts[inst * PHB_IREC + I_NCELLS]);
			res[s] = mode == 0 ? a / n : a; // mode 0: mean, 1: raw sum
		}
	}
	__syncthreads();
	if (threadIdx.x == 0) *counter = 0;
}

template <typename S, int D>
__global__ void __launch_bounds__(PHB_TILE) kSubtractMean(Dom<S, D> dom, S *__restrict__ x, int comps, const double *__restrict__ scratch) {
	__shared__ int32_t sB[PHB_BREC];
	int l0_, nc_;
	loadTile<S, D>(dom, sB, l0_, nc_);
	for (int j_ = 0; j_ < CPT; ++j_) {
	Cell c;
	if (!cellAt<D>(sB, l0_, nc_, j_, c)) return;
	const double *res = scratch + 8;
	const int inst = c.B[B_INST];
	for (int k = 0; k < comps; ++k) {
		const int64_t o = c.g + (int64_t)(comps - 1) * c.B[B_INSTOFF] + (int64_t)k * c.B[B_INSTN];
		x[o] = S(double(x[o]) - res[inst * comps + k]);
	}
	}
}

__global__ void kRmsFinish(const int32_t *insts, int ninst, int comps, const double *scratch, double *out) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= ninst) return;
	double s = 0;
	for (int k = 0; k < comps; ++k) s += scratch[8 + i * comps + k];
	out[i] = sqrt(s / (double(comps) * double(insts[i * PHB_IREC + I_NCELLS])));
}

// CSR pattern of the stencil: per cell the diagonal and the non-prescribed neighbours,
// ordered by column with ties kept in slot order, as PISO_build_matrix sorts its row
// (piso/advection.cu:269-288 with csr_rows.cuh:24-35).
template <int D>
__global__ void __launch_bounds__(PHB_TILE) kCsrRowSizes(Dom<double, D> dom, int32_t *rowsize) {
	__shared__ int32_t sB[PHB_BREC];
	int l0_, nc_;
	loadTile<double, D>(dom, sB, l0_, nc_);
	for (int j_ = 0; j_ < CPT; ++j_) {
	Cell c;
	if (!cellAt<D>(sB, l0_, nc_, j_, c)) return;
	int n = 2 * D + 1;
	for (int f = 0; f < 2 * D; ++f) if (atBound(c.B, f, c.p) && fType(c.B, f) == FT_FIXED) --n;
	rowsize[c.g] = n;
	}
}
template <int D>
__global__ void __launch_bounds__(PHB_TILE) kCsrPattern(Dom<double, D> dom, const int32_t *__restrict__ row, int32_t *col, int32_t *perm) {
	__shared__ int32_t sB[PHB_BREC];
	int l0_, nc_;
	loadTile<double, D>(dom, sB, l0_, nc_);
	for (int j_ = 0; j_ < CPT; ++j_) {
	Cell c;
	if (!cellAt<D>(sB, l0_, nc_, j_, c)) return;
	int64_t ci[2 * D + 1];
	ci[0] = c.g;
	for (int f = 0; f < 2 * D; ++f) ci[f + 1] = neighborIndex<double, D>(dom, c, f);
	int w = row[c.g];
	for (int it = 0; it < 2 * D + 1; ++it) {
		int best = -1;
		int64_t bv = INT64_MAX;
		for (int s = 0; s < 2 * D + 1; ++s) if (ci[s] >= 0 && ci[s] < bv) { bv = ci[s]; best = s; }
		if (best < 0) break;
		col[w] = (int32_t)bv;
		perm[w] = (int32_t)(best * dom.ncells + c.g);
		ci[best] = -1;
		++w;
	}
	}
}
template <typename T>
__global__ void kGather(int64_t n, const int32_t *__restrict__ perm, const T *__restrict__ src, T *__restrict__ dst) {
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) dst[i] = src[perm[i]];
}

// k_CoordsToTransforms (grid/grid_gen.cu:299-354): M from the differences of opposite face
// centres, Minv = adj(M)/det, written SoA.
template <typename S, int D>
__device__ __forceinline__ void writeTransform(const S (&M)[3][3], S *out, int64_t stride, int64_t idx) {
	S det, Mi[3][3] = {};
	if (D == 2) {
		det = M[0][0] * M[1][1] - M[1][0] * M[0][1];
		const S inv = S(1) / det;
		Mi[0][0] = M[1][1] * inv; Mi[0][1] = -M[0][1] * inv; Mi[1][0] = -M[1][0] * inv; Mi[1][1] = M[0][0] * inv;
	} else {
		det = M[0][0] * (M[1][1] * M[2][2] - M[2][1] * M[1][2]) - M[0][1] * (M[1][0] * M[2][2] - M[2][0] * M[1][2])
			+ M[0][2] * (M[1][0] * M[2][1] - M[2][0] * M[1][1]);
		const S inv = S(1) / det;
		Mi[0][0] = (M[1][1] * M[2][2] - M[2][1] * M[1][2]) * inv;
		Mi[0][1] = (M[0][2] * M[2][1] - M[0][1] * M[2][2]) * inv;
		Mi[0][2] = (M[0][1] * M[1][2] - M[0][2] * M[1][1]) * inv;
		Mi[1][0] = (M[1][2] * M[2][0] - M[1][0] * M[2][2]) * inv;
		Mi[1][1] = (M[0][0] * M[2][2] - M[0][2] * M[2][0]) * inv;
		Mi[1][2] = (M[1][0] * M[0][2] - M[0][0] * M[1][2]) * inv;
		Mi[2][0] = (M[1][0] * M[2][1] - M[2][0] * M[1][1]) * inv;
		Mi[2][1] = (M[2][0] * M[0][1] - M[0][0] * M[2][1]) * inv;
		Mi[2][2] = (M[0][0] * M[1][1] - M[1][0] * M[0][1]) * inv;
	}
	for (int i = 0; i < D; ++i)
		for (int k = 0; k < D; ++k) {
			out[(i * D + k) * stride + idx] = M[i][k];
			out[(D * D + i * D + k) * stride + idx] = Mi[i][k];
		}
	out[(2 * D * D) * stride + idx] = det;
}

template <typename S, int D>
__global__ void kCellMetrics(int nx, int ny, int nz, const S *__restrict__ coords, S *out, int64_t stride) {
	const int64_t n = (int64_t)nx * ny * (D > 2 ? nz : 1);
	const int vx = nx + 1, vy = ny + 1;
	const int64_t vstride = (int64_t)vx * vy * (D > 2 ? nz + 1 : 1);
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
		const int x = int(i % nx), y = int((i / nx) % ny), z = int(i / ((int64_t)nx * ny));
		S fc[6][3] = {};
		for (int v = 0; v < (1 << D); ++v) {
			const int px = x + (v & 1), py = y + ((v & 2) != 0), pz = z + ((v & 4) != 0);
			for (int f = 0; f < D; ++f) {
				const int up = (v & (1 << f)) != 0;
				for (int k = 0; k < D; ++k) fc[f * 2 + up][k] += coords[k * vstride + ((int64_t)pz * vy + py) * vx + px];
			}
		}
		const S norm = S(1) / S(1 << (D - 1));
		S M[3][3] = {};
		for (int i2 = 0; i2 < D; ++i2)
			for (int k = 0; k < D; ++k) M[i2][k] = fc[k * 2 + 1][i2] * norm - fc[k * 2][i2] * norm;
		writeTransform<S, D>(M, out, stride, i);
	}
}

// k_CoordsToFaceTransforms (grid/grid_gen.cu:398-490) evaluated at the faces of one block
// side, as Block::GetFaceTransformBoundarySlice slices it (domain/block.cpp:790-816)
template <typename S, int D>
__global__ void kFaceMetrics(int nx, int ny, int nz, const S *__restrict__ coords, int face, S *out, int64_t stride) {
	const int vsz[3] = {nx + 1, ny + 1, D > 2 ? nz + 1 : 1};
	const int csz[3] = {nx, ny, D > 2 ? nz : 1};
	const int64_t vstride = (int64_t)vsz[0] * vsz[1] * vsz[2];
	const int dim = face >> 1;
	int fsz[3] = {csz[0], csz[1], csz[2]};
	fsz[dim] = 1;
	const int64_t n = (int64_t)fsz[0] * fsz[1] * fsz[2];
	const int numFaceVertices = 1 << (D - 1);
	const int numEdgeVertices = 1 << (D - 2);
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
		int pos[3] = {int(i % fsz[0]), int((i / fsz[0]) % fsz[1]), int(i / ((int64_t)fsz[0] * fsz[1]))};
		pos[dim] = (face & 1) ? csz[dim] : 0;
		S t[3][3] = {};
		S normWeight = 0.5;
		for (int up = 0; up < 2; ++up) {
			const int faceSign = up * 2 - 1;
			const bool atB = up ? pos[dim] == vsz[dim] - 1 : pos[dim] == 0;
			int fp[3] = {pos[0], pos[1], pos[2]};
			if (!atB) fp[dim] += faceSign; else normWeight = 1.0;
			for (int v = 0; v < numFaceVertices; ++v) {
				int vp[3] = {fp[0], fp[1], fp[2]};
				for (int k2 = 1; k2 < D; ++k2) vp[(dim + k2) % D] += (v & k2) != 0;
				for (int k = 0; k < D; ++k) t[k][dim] += coords[k * vstride + ((int64_t)vp[2] * vsz[1] + vp[1]) * vsz[0] + vp[0]] * S(faceSign);
			}
		}
		normWeight /= S(numFaceVertices);
		for (int k = 0; k < D; ++k) t[k][dim] *= normWeight;
		const S tNorm = S(1) / S(numEdgeVertices);
		for (int kk = 1; kk < D; ++kk) {
			const int tDim = (dim + kk) % D;
			for (int v = 0; v < numFaceVertices; ++v) {
				int vp[3] = {pos[0], pos[1], pos[2]};
				for (int k2 = 1; k2 < D; ++k2) vp[(dim + k2) % D] += (v & k2) != 0;
				const S ts = (v & kk) ? S(1) : S(-1);
				for (int k = 0; k < D; ++k) t[k][tDim] += coords[k * vstride + ((int64_t)vp[2] * vsz[1] + vp[1]) * vsz[0] + vp[0]] * ts;
			}
			for (int k = 0; k < D; ++k) t[k][tDim] *= tNorm;
		}
		writeTransform<S, D>(t, out, stride, i);
	}
}

} // namespace phb

using namespace phb;

#define PHB_DISPATCH(DOM, ...)                                                                     \
	do {                                                                                           \
		if ((DOM)->dims == 2 && (DOM)->dtype == PHB_F64) { using S = double; constexpr int D = 2; __VA_ARGS__; } \
		else if ((DOM)->dims == 3 && (DOM)->dtype == PHB_F64) { using S = double; constexpr int D = 3; __VA_ARGS__; } \
		else if ((DOM)->dims == 2 && (DOM)->dtype == PHB_F32) { using S = float; constexpr int D = 2; __VA_ARGS__; } \
		else if ((DOM)->dims == 3 && (DOM)->dtype == PHB_F32) { using S = float; constexpr int D = 3; __VA_ARGS__; } \
		else return setError(PHB_ERR_ARG, "unsupported dims/dtype");                                \
	} while (0)

extern "C" const char *phb_last_error(void) { return tlError.c_str(); }
extern "C" int phb_version(void) { return 1; }

extern "C" int phb_subtract_mean(const phb_domain *dom, void *x, int comps, double *scratch, phb_stream stream) {
	if (!dom || !x || !scratch || comps < 1 || comps > 3) return setError(PHB_ERR_ARG, "phb_subtract_mean: bad argument");
	if (dom->ntiles == 0) return PHB_OK;
	cudaStream_t s = (cudaStream_t)stream;
	PHB_DISPATCH(dom, {
		kInstanceSums<S, D, 1><<<dom->ntiles, PHB_TILE, 0, s>>>(Dom<S, D>(*dom), (const S *)x, comps, scratch, 0);
		kSubtractMean<S, D><<<dom->ntiles, PHB_TILE, 0, s>>>(Dom<S, D>(*dom), (S *)x, comps, scratch);
	});
	return checkLaunch("phb_subtract_mean");
}

extern "C" int64_t phb_scratch_doubles(const phb_domain *dom, int comps) {
	if (!dom) return -1;
	return 8 + (int64_t)dom->ninst * comps + (int64_t)dom->ntiles * comps;
}

extern "C" int phb_rms(const phb_domain *dom, const void *v, int comps, double *scratch, double *out, phb_stream stream) {
	if (!dom || !v || !scratch || !out || comps < 1 || comps > 3) return setError(PHB_ERR_ARG, "phb_rms: bad argument");
	if (dom->ntiles == 0) return PHB_OK;
	cudaStream_t s = (cudaStream_t)stream;
	PHB_DISPATCH(dom, kInstanceSums<S, D, 2><<<dom->ntiles, PHB_TILE, 0, s>>>(Dom<S, D>(*dom), (const S *)v, comps, scratch, 1));
	const int rc = checkLaunch("phb_rms sums");
	if (rc) return rc;
	kRmsFinish<<<(dom->ninst + 127) / 128, 128, 0, s>>>(dom->insts, dom->ninst, comps, scratch, out);
	return checkLaunch("phb_rms finish");
}

extern "C" int phb_csr_row_sizes(const phb_domain *dom, int32_t *rowsize, phb_stream stream) {
	if (!dom || !rowsize) return setError(PHB_ERR_ARG, "phb_csr_row_sizes: null argument");
	if (dom->ntiles == 0) return PHB_OK;
	cudaStream_t s = (cudaStream_t)stream;
	if (dom->dims == 2) kCsrRowSizes<2><<<dom->ntiles, PHB_TILE, 0, s>>>(Dom<double, 2>(*dom), rowsize);
	else if (dom->dims == 3) kCsrRowSizes<3><<<dom->ntiles, PHB_TILE, 0, s>>>(Dom<double, 3>(*dom), rowsize);
	else return setError(PHB_ERR_ARG, "dims");
	return checkLaunch("kCsrRowSizes");
}
extern "C" int phb_csr_pattern(const phb_domain *dom, const int32_t *row, int32_t *col, int32_t *perm, phb_stream stream) {
	if (!dom || !row || !col || !perm) return setError(PHB_ERR_ARG, "phb_csr_pattern: null argument");
	if (dom->ntiles == 0) return PHB_OK;
	cudaStream_t s = (cudaStream_t)stream;
	if (dom->dims == 2) kCsrPattern<2><<<dom->ntiles, PHB_TILE, 0, s>>>(Dom<double, 2>(*dom), row, col, perm);
	else if (dom->dims == 3) kCsrPattern<3><<<dom->ntiles, PHB_TILE, 0, s>>>(Dom<double, 3>(*dom), row, col, perm);
	else return setError(PHB_ERR_ARG, "dims");
	return checkLaunch("kCsrPattern");
}
extern "C" int phb_csr_gather(int dtype, int64_t nnz, const int32_t *perm, const void *stencil, void *value, phb_stream stream) {
	if (!perm || !stencil || !value || nnz < 0) return setError(PHB_ERR_ARG, "phb_csr_gather: bad argument");
	if (nnz == 0) return PHB_OK;
	const int grid = (int)std::min<int64_t>((nnz + 255) / 256, 148 * 16);
	cudaStream_t s = (cudaStream_t)stream;
	if (dtype == PHB_F64) kGather<double><<<grid, 256, 0, s>>>(nnz, perm, (const double *)stencil, (double *)value);
	else if (dtype == PHB_F32) kGather<float><<<grid, 256, 0, s>>>(nnz, perm, (const float *)stencil, (float *)value);
	else return setError(PHB_ERR_ARG, "dtype");
	return checkLaunch("kGather");
}

extern "C" int phb_cell_metrics(int dims, int dtype, int nx, int ny, int nz, const void *coords, void *cell_out, int64_t stride, phb_stream stream) {
	if (!coords || !cell_out || nx < 1 || ny < 1 || (dims == 3 && nz < 1)) return setError(PHB_ERR_ARG, "phb_cell_metrics: bad argument");
	const int64_t n = (int64_t)nx * ny * (dims > 2 ? nz : 1);
	const int grid = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
	cudaStream_t s = (cudaStream_t)stream;
	if (dims == 2 && dtype == PHB_F64) kCellMetrics<double, 2><<<grid, 256, 0, s>>>(nx, ny, nz, (const double *)coords, (double *)cell_out, stride);
	else if (dims == 3 && dtype == PHB_F64) kCellMetrics<double, 3><<<grid, 256, 0, s>>>(nx, ny, nz, (const double *)coords, (double *)cell_out, stride);
	else if (dims == 2 && dtype == PHB_F32) kCellMetrics<float, 2><<<grid, 256, 0, s>>>(nx, ny, nz, (const float *)coords, (float *)cell_out, stride);
	else if (dims == 3 && dtype == PHB_F32) kCellMetrics<float, 3><<<grid, 256, 0, s>>>(nx, ny, nz, (const float *)coords, (float *)cell_out, stride);
	else return setError(PHB_ERR_ARG, "phb_cell_metrics: dims/dtype");
	return checkLaunch("kCellMetrics");
}
extern "C" int phb_face_metrics(int dims, int dtype, int nx, int ny, int nz, const void *coords, int face, void *face_out, int64_t stride, phb_stream stream) {
	if (!coords || !face_out || face < 0 || face >= 2 * dims) return setError(PHB_ERR_ARG, "phb_face_metrics: bad argument");
	cudaStream_t s = (cudaStream_t)stream;
	if (dims == 2 && dtype == PHB_F64) kFaceMetrics<double, 2><<<64, 256, 0, s>>>(nx, ny, nz, (const double *)coords, face, (double *)face_out, stride);
	else if (dims == 3 && dtype == PHB_F64) kFaceMetrics<double, 3><<<64, 256, 0, s>>>(nx, ny, nz, (const double *)coords, face, (double *)face_out, stride);
	else if (dims == 2 && dtype == PHB_F32) kFaceMetrics<float, 2><<<64, 256, 0, s>>>(nx, ny, nz, (const float *)coords, face, (float *)face_out, stride);
	else if (dims == 3 && dtype == PHB_F32) kFaceMetrics<float, 3><<<64, 256, 0, s>>>(nx, ny, nz, (const float *)coords, face, (float *)face_out, stride);
	else return setError(PHB_ERR_ARG, "phb_face_metrics: dims/dtype");
	return checkLaunch("kFaceMetrics");
}
