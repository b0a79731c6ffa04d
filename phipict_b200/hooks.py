"""Ordered callback points of a PISO step (phiPICT core/hooks.py:26-205)."""
from __future__ import annotations

from enum import Enum
from typing import Any, Callable, Mapping


class Hook(str, Enum):
    """A point of a PISO step at which the registered callbacks run, in step order.
    Callbacks receive the keyword arguments ``domain``, ``local_step``, ``time_step``,
    ``total_step`` and ``total_time``."""
    PRE = "PRE"
    POST_SCALAR_SETUP = "POST_SCALAR_SETUP"
    PRE_VELOCITY_SETUP = "PRE_VELOCITY_SETUP"
    POST_VELOCITY_SETUP = "POST_VELOCITY_SETUP"
    POST_PREDICTION = "POST_PREDICTION"
    POST_PRESSURE_SETUP = "POST_PRESSURE_SETUP"
    POST_PRESSURE_RESULT = "POST_PRESSURE_RESULT"
    POST_PRESSURE_NON_ORTHO = "POST_PRESSURE_NON_ORTHO"
    POST_VELOCITY_CORRECTION = "POST_VELOCITY_CORRECTION"
    POST = "POST"

    def __str__(self) -> str:
        return self.value

    @classmethod
    def parse(cls, name: "str | Hook") -> "Hook":
        try:
            return cls(name)
        except ValueError:
            valid = ", ".join(h.value for h in cls)
            raise ValueError(f"Unknown hook {name!r}; valid hooks: {valid}.") from None


HookFn = Callable[..., Any]


class Hooks:
    """The callbacks of a simulation per :class:`Hook`, in registration order."""

    def __init__(self, callbacks: "Hooks | Mapping[Hook | str, Any] | None" = None) -> None:
        self._callbacks: dict[Hook, list[HookFn]] = {}
        if callbacks is None:
            return
        items = callbacks._callbacks.items() if isinstance(callbacks, Hooks) else callbacks.items()
        for hook, fns in items:
            if fns is None:
                continue
            if callable(fns):
                fns = [fns]
            for fn in fns:
                if fn is not None:
                    self.append(hook, fn)

    @classmethod
    def coerce(cls, hooks) -> "Hooks":
        return hooks if isinstance(hooks, Hooks) else cls(hooks)

    def append(self, hook: "Hook | str", fn: HookFn) -> "Hooks":
        self._callbacks.setdefault(Hook.parse(hook), []).append(fn)
        return self

    def prepend(self, hook: "Hook | str", fn: HookFn) -> "Hooks":
        self._callbacks.setdefault(Hook.parse(hook), []).insert(0, fn)
        return self

    def run(self, hook: Hook, **kwargs: Any) -> None:
        for fn in self._callbacks.get(hook, ()):
            fn(**kwargs)

    def has(self, hook: Hook) -> bool:
        return bool(self._callbacks.get(hook))

    def __bool__(self) -> bool:
        return any(self._callbacks.values())

    def __len__(self) -> int:
        return sum(len(v) for v in self._callbacks.values())
