"""``Packing``: the stateful API of RCPGenerator on the B200 engine.

Same constructor arguments, attributes, methods, state flags and results as
the reference class (python_code/python/python/rcpgenerator/_wrapper.py:28-628),
so code written against ``rcpgenerator.Packing`` runs unchanged. One keyword is
added: ``engine`` = "graph" (default, GPU-resident controller) or "exact"
(host controller, one-thread reduction order). Rendering and animation need
matplotlib and are not part of this engine.
"""

from __future__ import annotations

import math
from copy import deepcopy
from typing import Any

from . import _api


def _container_fraction(walls) -> float:
    """Fraction of the bounding box a t-ball container fills (walls[0] = -t),
    1.0 otherwise; phi is reported against the container (_wrapper.py:15-23)."""
    t = -int(walls[0]) if (walls and int(walls[0]) < 0) else 0
    if t < 2:
        return 1.0
    return math.pi ** (t / 2.0) / math.gamma(t / 2.0 + 1.0) * (0.5 ** t)


class Packing:
    _INIT_KEYS = {"phi", "N", "Ndim", "box", "walls", "fix_height", "dist"}
    _PACK_KEYS = {"box", "walls", "neighbor_max", "seed", "fix_height"}
    _REALIZED_STATE_KEYS = {"positions", "diameters"}
    _RESULT_KEYS = {"steps", "phi_final", "max_min_dist", "force_magnitude", "phi_history",
                    "force_history", "energy_history"}
    _RESULT_LISTS = ("phi_history", "force_history", "energy_history", "max_overlap_history",
                     "mu_flag_history", "mu_history", "alpha_history")
    _TRAJ = ("positions", "diameters", "steps", "phi", "force", "energy", "max_min_dist")

    # ---- construction ----------------------------------------------------
    def __init__(self, **kwargs: Any) -> None:
        self._set_flags(initialized=False, packed=False, needs_initialize=True, needs_pack=True)
        object.__setattr__(self, "_mutating_internal_state", True)
        self.verbose = kwargs.pop("verbose", False)
        self.phi = kwargs.pop("phi", 0.05)
        self.N = kwargs.pop("N", 0)
        self.Ndim = kwargs.pop("Ndim", 0)
        self.box = deepcopy(kwargs.pop("box", []))
        self.walls = deepcopy(kwargs.pop("walls", [0] * len(self.box) if self.box else []))
        self.fix_height = kwargs.pop("fix_height", False)
        self.dist = deepcopy(kwargs.pop("dist", {"type": "mono", "d": 1.0}))
        self.neighbor_max = kwargs.pop("neighbor_max", 0)
        self.seed = kwargs.pop("seed", 0)
        self.engine = kwargs.pop("engine", "graph")
        self.positions = []
        self.diameters = []
        self._reset_result_fields()
        self._reset_trajectory_fields()
        if kwargs:
            raise TypeError(f"Unexpected keyword argument(s): {', '.join(sorted(kwargs))}")
        object.__setattr__(self, "_mutating_internal_state", False)
        self.initialize()

    @classmethod
    def from_dict(cls, data: dict[str, Any]) -> "Packing":
        init = deepcopy(data.get("init_config", {}))
        pack = deepcopy(data.get("pack_config", {}))
        state = deepcopy(data.get("realized_state", {}))
        final = deepcopy(data.get("final_result", {}))
        traj = deepcopy(data.get("trajectory", {}))
        status = deepcopy(data.get("status", {}))
        obj = cls.__new__(cls)
        obj._set_flags(initialized=False, packed=False, needs_initialize=True, needs_pack=True)
        object.__setattr__(obj, "_mutating_internal_state", True)
        obj.verbose = init.pop("verbose", pack.pop("verbose", False))
        obj.phi = init.get("phi", 0.05)
        obj.N = init.get("N", 0)
        obj.Ndim = init.get("Ndim", 0)
        obj.box = deepcopy(init.get("box", pack.get("box", [])))
        obj.walls = deepcopy(init.get("walls", pack.get("walls", [])))
        obj.fix_height = init.get("fix_height", pack.get("fix_height", False))
        obj.dist = deepcopy(init.get("dist", {}))
        obj.neighbor_max = pack.get("neighbor_max", 0)
        obj.seed = pack.get("seed", 0)
        obj.engine = pack.get("engine", "graph")
        obj.positions = deepcopy(state.get("positions", []))
        obj.diameters = deepcopy(state.get("diameters", []))
        obj._reset_result_fields()
        obj.steps = final.get("steps", 0)
        obj.phi_final = final.get("phi_final")
        obj.max_min_dist = final.get("max_min_dist")
        obj.force_magnitude = final.get("force_magnitude")
        for k in ("phi_history", "force_history", "energy_history"):
            setattr(obj, k, deepcopy(final.get(k, [])))
        for k in cls._TRAJ:
            setattr(obj, "trajectory_" + k, deepcopy(traj.get(k, [])))
        initialized = bool(status.get("initialized", bool(obj.positions) and bool(obj.diameters)))
        packed = bool(status.get("packed", bool(obj.steps)))
        obj._set_flags(
            initialized=initialized,
            packed=packed,
            needs_initialize=bool(status.get("needs_initialize", not initialized)),
            needs_pack=bool(status.get("needs_pack", not packed)),
        )
        object.__setattr__(obj, "_mutating_internal_state", False)
        return obj

    # ---- state bookkeeping -----------------------------------------------
    def _set_flags(self, **flags: bool) -> None:
        for k, v in flags.items():
            object.__setattr__(self, "_" + k, v)

    def _reset_result_fields(self) -> None:
        self.steps = 0
        self.phi_final = None
        self.max_min_dist = None
        self.force_magnitude = None
        for k in self._RESULT_LISTS:
            setattr(self, k, [])

    def _reset_trajectory_fields(self) -> None:
        for k in self._TRAJ:
            setattr(self, "trajectory_" + k, [])

    def __setattr__(self, name: str, value: Any) -> None:
        object.__setattr__(self, name, value)
        if name.startswith("_") or getattr(self, "_mutating_internal_state", False):
            return
        if name in self._INIT_KEYS:
            self._set_flags(needs_initialize=True, needs_pack=True, packed=False)
        elif name in self._PACK_KEYS or name in self._REALIZED_STATE_KEYS:
            self._set_flags(needs_pack=True, packed=False)

    def __repr__(self) -> str:
        return (f"Packing(N={self.N}, Ndim={self.Ndim}, initialized={self._initialized}, "
                f"packed={self._packed}, needs_initialize={self._needs_initialize}, "
                f"needs_pack={self._needs_pack})")

    @property
    def needs_initialize(self) -> bool:
        return self._needs_initialize

    @property
    def needs_pack(self) -> bool:
        return self._needs_pack

    @property
    def initialized(self) -> bool:
        return self._initialized

    @property
    def packed(self) -> bool:
        return self._packed

    def _log(self, message: str) -> None:
        if self.verbose:
            print(message)

    def _internal(self):
        obj = self

        class _Guard:
            def __enter__(self_inner):
                object.__setattr__(obj, "_mutating_internal_state", True)

            def __exit__(self_inner, *exc):
                object.__setattr__(obj, "_mutating_internal_state", False)
                return False

        return _Guard()

    # ---- dicts exchanged with the engine -----------------------------------
    def _collect_init_config(self) -> dict[str, Any]:
        return {"phi": self.phi, "N": self.N, "Ndim": self.Ndim, "box": deepcopy(self.box),
                "walls": deepcopy(self.walls), "fix_height": self.fix_height,
                "dist": deepcopy(self.dist), "seed": self.seed}

    def _collect_pack_input(self) -> dict[str, Any]:
        return {"positions": deepcopy(self.positions), "diameters": deepcopy(self.diameters)}

    def _collect_pack_config(self) -> dict[str, Any]:
        return {"box": deepcopy(self.box), "walls": deepcopy(self.walls),
                "neighbor_max": self.neighbor_max, "seed": self.seed,
                "fix_height": self.fix_height, "engine": self.engine}

    def _current_phi(self) -> float:
        if not self.positions or not self.diameters or not self.box:
            raise ValueError("Current realized state is unavailable")
        # plain left-to-right sums as the reference (WRP:267-280); Python's
        # sum() of floats is compensated and rounds differently
        box_volume = 1.0
        for length in self.box:
            box_volume *= length
        coeff = math.pi ** (self.Ndim / 2.0) / math.gamma(self.Ndim / 2.0 + 1.0)
        volume = 0.0
        for d in self.diameters:
            volume += coeff * (d / 2.0) ** self.Ndim
        modifier = 1.0
        if self.walls and self.walls[0] < 0:
            t = -self.walls[0]
            modifier = math.pi ** (t / 2.0) / math.gamma(t / 2.0 + 1.0) * (0.5 ** t)
        return volume / box_volume / modifier

    def _apply_initializer_result(self, result: dict[str, Any]) -> None:
        with self._internal():
            self.positions = result["positions"]
            self.diameters = result["diameters"]
            self.box = result["box"]
            self.walls = result["walls"]
            self._reset_result_fields()
        self._set_flags(initialized=True, needs_initialize=False, needs_pack=True, packed=False)

    def _apply_packing_result(self, result: dict[str, Any]) -> None:
        cf = _container_fraction(result["walls"])
        with self._internal():
            self.positions = result["positions"]
            self.diameters = result["diameters"]
            self.box = result["box"]
            self.walls = result["walls"]
            self.steps = result["steps"]
            self.phi_final = result["phi"] / cf
            self.max_min_dist = result["max_min_dist"]
            self.force_magnitude = result["force_magnitude"]
            self.phi_history = ([v / cf for v in result["phi_history"]] if cf != 1.0
                                else result["phi_history"])
            self.force_history = result["force_history"]
            self.energy_history = result["energy_history"]
            self.max_overlap_history = result.get("max_overlap_history", [])
            self.mu_flag_history = result.get("mu_flag_history", [])
            self.mu_history = result.get("mu_history", [])
            self.alpha_history = result.get("alpha_history", [])
        self._set_flags(packed=True, needs_pack=False)

    def _apply_trajectory(self, trace: dict[str, Any]) -> None:
        with self._internal():
            for k in self._TRAJ:
                setattr(self, "trajectory_" + k, trace.get(k, []))

    def _execute_packing(self, *, verbose: bool, progress_interval: int,
                         capture_trajectory: bool, trajectory_interval: int,
                         options: dict[str, Any] | None = None) -> dict[str, Any]:
        with self._internal():
            self._reset_trajectory_fields()
        if verbose:
            print("rcpgenerator: running packing")
        if verbose or capture_trajectory or options:
            def on_progress(update: dict[str, Any]) -> None:
                if verbose:
                    print(f"step={update['step']} phi={update['phi']:.6f} "
                          f"force={update['force_magnitude']:.6g} energy={update['energy']:.6g}")

            observed = _api.run_packing_observed(
                self._collect_pack_input(), self._collect_pack_config(),
                progress_interval if verbose else 0, capture_trajectory,
                trajectory_interval if capture_trajectory else 0,
                on_progress if verbose else None, options or {})
            result = observed["result"]
            self._apply_packing_result(result)
            self._apply_trajectory(observed["trace"])
        else:
            result = _api.run_packing(self._collect_pack_input(), self._collect_pack_config())
            self._apply_packing_result(result)
        if verbose:
            print("rcpgenerator: packing complete")
        return result

    # ---- public API ------------------------------------------------------
    def initialize(self) -> dict[str, Any]:
        self._log("rcpgenerator: initializing particles")
        result = _api.initialize_particles(self._collect_init_config())
        self._apply_initializer_result(result)
        self._log("rcpgenerator: initialization complete")
        return result

    def pack(self, verbose: bool | None = None, progress_interval: int = 1000,
             capture_trajectory: bool = False, trajectory_interval: int = 1000) -> dict[str, Any]:
        eff = self.verbose if verbose is None else verbose
        if self._needs_initialize or not self._initialized:
            if eff:
                print("rcpgenerator: initialization required before packing")
            self.initialize()
        elif self._needs_pack and eff:
            print("rcpgenerator: rerunning packing on current realized state")
        return self._execute_packing(verbose=eff, progress_interval=progress_interval,
                                     capture_trajectory=capture_trajectory,
                                     trajectory_interval=trajectory_interval)

    def relax(self, n_steps: int, mu: float | None = None, fix_diameter: bool = False,
              target_phi: float | None = None, verbose: bool = False, progress_interval: int = 1000,
              capture_trajectory: bool = False, trajectory_interval: int = 1000) -> dict[str, Any]:
        if n_steps <= 0:
            raise ValueError("n_steps must be positive")
        if target_phi is not None and fix_diameter:
            raise ValueError("target_phi cannot be combined with fix_diameter=True")
        if self._needs_initialize or not self._initialized:
            if verbose:
                print("rcpgenerator: initialization required before relaxation")
            self.initialize()
        elif self._needs_pack and verbose:
            print("rcpgenerator: relaxing current realized state")
        options: dict[str, Any] = {"max_steps": int(n_steps), "fix_diameter": bool(fix_diameter)}
        if mu is not None:
            options["mu"] = float(mu)
        if target_phi is not None:
            options["target_phi"] = float(target_phi)
        return self._execute_packing(verbose=verbose, progress_interval=progress_interval,
                                     capture_trajectory=capture_trajectory,
                                     trajectory_interval=trajectory_interval, options=options)

    def render(self, *args: Any, **kwargs: Any):
        raise NotImplementedError("rendering (matplotlib) is not part of the B200 engine")

    savefig = render
    show_packing = render
    animate_2d = render

    def summary(self) -> str:
        return (f"Packing summary: N={self.N}, Ndim={self.Ndim}, phi={self.phi}, "
                f"initialized={self.initialized}, packed={self.packed}, "
                f"needs_initialize={self.needs_initialize}, needs_pack={self.needs_pack}, "
                f"phi_final={self.phi_final}, steps={self.steps}, "
                f"force_magnitude={self.force_magnitude}, "
                f"trajectory_samples={len(self.trajectory_steps)}")

    def reset(self) -> None:
        with self._internal():
            self.positions = []
            self.diameters = []
            self._reset_result_fields()
            self._reset_trajectory_fields()
        self._set_flags(initialized=False, packed=False, needs_initialize=True, needs_pack=True)

    def _mark_realized_state_updated(self) -> None:
        with self._internal():
            self._reset_result_fields()
            self._reset_trajectory_fields()
        self._set_flags(needs_pack=True, packed=False)

    def update_phi(self, target_phi: float) -> float:
        if target_phi <= 0:
            raise ValueError("target_phi must be positive")
        current = self._current_phi()
        exponent = self.Ndim - 1 if self.fix_height else self.Ndim
        scale = (target_phi / current) ** (1.0 / exponent)
        with self._internal():
            self.diameters = [d * scale for d in self.diameters]
            if self.fix_height:
                box = list(self.box)
                box[self.Ndim - 1] *= scale
                self.box = box
                self.positions = [[c * scale if k == self.Ndim - 1 else c for k, c in enumerate(p)]
                                  for p in self.positions]
        self._mark_realized_state_updated()
        return self._current_phi()

    def update_box(self, box: list[float]) -> list[float]:
        if len(box) != self.Ndim:
            raise ValueError("box length must match Ndim")
        if not self.positions or not self.diameters or not self.box:
            raise ValueError("Current realized state is unavailable")
        old = list(self.box)
        new = [float(v) for v in box]
        old_v, new_v = math.prod(old), math.prod(new)
        if old_v <= 0 or new_v <= 0:
            raise ValueError("box dimensions must be positive")
        dscale = (new_v / old_v) ** (1.0 / self.Ndim)
        pscale = [new[k] / old[k] for k in range(self.Ndim)]
        with self._internal():
            self.box = new
            self.positions = [[c * pscale[k] for k, c in enumerate(p)] for p in self.positions]
            self.diameters = [d * dscale for d in self.diameters]
        self._mark_realized_state_updated()
        return list(self.box)

    def update_height(self, height: float) -> list[float]:
        box = list(self.box)
        if not box:
            raise ValueError("Current box is unavailable")
        box[self.Ndim - 1] = float(height)
        return self.update_box(box)

    def copy(self) -> "Packing":
        return type(self).from_dict(self.to_dict())

    def clone(self) -> "Packing":
        return self.copy()

    def to_dict(self) -> dict[str, Any]:
        return {
            "init_config": self._collect_init_config(),
            "pack_config": self._collect_pack_config(),
            "realized_state": self._collect_pack_input(),
            "final_result": {
                "steps": self.steps, "phi_final": self.phi_final,
                "max_min_dist": self.max_min_dist, "force_magnitude": self.force_magnitude,
                "phi_history": deepcopy(self.phi_history),
                "force_history": deepcopy(self.force_history),
                "energy_history": deepcopy(self.energy_history),
            },
            "trajectory": {k: deepcopy(getattr(self, "trajectory_" + k)) for k in self._TRAJ},
            "status": {"initialized": self._initialized, "packed": self._packed,
                       "needs_initialize": self._needs_initialize, "needs_pack": self._needs_pack},
        }
