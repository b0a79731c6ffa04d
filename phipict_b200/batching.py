"""Per-environment state of a batched domain (phiPICT batching.py:178-320).

Per-environment adaptive substeps advance every environment of a batch by its own CFL-bound
substeps; an environment that has covered its time step still runs through the batch's
remaining substeps, and its state is put back afterwards from an :class:`EnvStateSnapshot`.
Every field here is one flat device buffer with a slice per environment, so a snapshot is an
index_select of those rows and a restore is an index_copy.
"""
from __future__ import annotations

from typing import Callable, Sequence

import torch


class EnvStateSnapshot:
    """State of some environments of a batched domain, to undo a substep for them: the block
    fields (velocity, pressure, passive scalar, potential), the solution vectors (the next
    solves' initial guesses and the potential the Lorentz force uses), the velocity source (a
    hook accumulates the Lorentz force into it) and `extra` flat per-environment tensors."""

    def __init__(self, domain, env_idx: torch.Tensor,
                 extra: Sequence[Callable[[], torch.Tensor | None]] = ()) -> None:
        self._domain = domain
        self._batch = domain.getBatchSize()
        self._idx = env_idx.to(device=domain.getDevice(), dtype=torch.long).reshape(-1)
        getters: list[Callable[[], torch.Tensor | None]] = [
            lambda: domain._u_block,
            lambda: domain._p_block,
            lambda: getattr(domain, "_phi_block", None),
            lambda: getattr(domain, "_epot_block", None),
            lambda: domain.velocityResult,
            lambda: domain.pressureResult,
            lambda: getattr(domain, "scalarResult", None),
            lambda: getattr(domain, "epotResult", None),
            lambda: domain._src if getattr(domain, "_src", None) is not None and domain._src.shape[0] == self._batch else None,
            *extra,
        ]
        self._fields: list[tuple[Callable[[], torch.Tensor | None], torch.Tensor]] = []
        with torch.no_grad():
            for g in getters:
                t = g()
                if t is None or t.numel() == 0:
                    continue
                self._fields.append((g, self._rows(t).index_select(0, self._idx).clone()))

    def _rows(self, t: torch.Tensor) -> torch.Tensor:
        if t.numel() % self._batch:
            raise RuntimeError("a per-environment tensor must hold one equal slice per environment")
        return t.reshape(self._batch, -1)

    def restore(self) -> None:
        """Write the saved rows back (tensors are read through their getters again)."""
        with torch.no_grad():
            for g, saved in self._fields:
                t = g()
                if t is None:
                    continue
                self._rows(t).index_copy_(0, self._idx, saved)


__all__ = ["EnvStateSnapshot"]
