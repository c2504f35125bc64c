"""ctypes binding of the C ABI (include/nepheline_b200.h).

Loads lib/libnepheline_b200.so and fails loudly when it is missing: there is no other
implementation of the solver stage in this package.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

from . import abi

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libnepheline_b200.so"
_lib = None

_u32 = ctypes.c_uint32
_vp = ctypes.c_void_p


class SolverError(RuntimeError):
    def __init__(self, code: int, what: str):
        super().__init__(f"{what}: {abi.RESULT_NAMES.get(code, code)}")
        self.code = code


def lib() -> ctypes.CDLL:
    """The shared library, with its signatures declared."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: build it with python -m nepheline_b200.build")
    L = ctypes.CDLL(str(LIB_PATH))
    P = ctypes.POINTER
    sig = {
        "nph_gpu_solver_create": (ctypes.c_int32, [P(abi.SolverDesc), P(_vp)]),
        "nph_gpu_solver_destroy": (None, [_vp]),
        "nph_gpu_phys_solve": (ctypes.c_int32, [_vp, P(abi.WorldParams), ctypes.c_float,
                                                P(abi.WorldView)]),
        "nph_gpu_phys_solve_packed": (ctypes.c_int32, [_vp, P(abi.WorldParams), ctypes.c_float,
                                                       P(abi.PackedInput), P(abi.PackedOutput)]),
        "nph_gpu_world_upload": (ctypes.c_int32, [_vp, P(abi.WorldView)]),
        "nph_gpu_world_step_async": (ctypes.c_int32, [_vp, P(abi.WorldParams), ctypes.c_float,
                                                      _u32]),
        "nph_gpu_world_download": (ctypes.c_int32, [_vp, P(abi.WorldView)]),
        "nph_gpu_solver_synchronize": (ctypes.c_int32, [_vp]),
        "nph_gpu_solver_stats": (ctypes.c_int32, [_vp, P(abi.StepStats)]),
        "nph_gpu_solver_stream": (_vp, [_vp]),
        "nph_gpu_solver_set_memory_limit": (ctypes.c_int32, [_vp, ctypes.c_uint64]),
        "nph_gpu_solver_set_wait_injection": (ctypes.c_int32, [_vp, _u32]),
        "nph_gpu_batch_set_pass_config": (ctypes.c_int32, [_vp, _u32, _u32]),
        "nph_gpu_solver_memory": (ctypes.c_uint64, [_vp]),
        "nph_gpu_graph_color": (ctypes.c_int32, [_vp, _vp, _vp, _vp, _u32, _u32, _vp, _vp]),
        "nph_gpu_version": (ctypes.c_char_p, []),
        "nph_gpu_world_profile_step": (ctypes.c_int32, [_vp, P(abi.WorldParams), ctypes.c_float,
                                                        P(abi.KernelTime), _u32, P(_u32)]),
        "nph_gpu_solver_set_pass_config": (ctypes.c_int32, [_vp, _u32, _u32]),
        "nph_gpu_mlp_create": (ctypes.c_int32, [ctypes.c_int32, ctypes.c_uint64, P(_vp)]),
        "nph_gpu_mlp_destroy": (None, [_vp]),
        "nph_gpu_mlp_set_weights": (ctypes.c_int32, [_vp, _vp]),
        "nph_gpu_mlp_get_weights": (ctypes.c_int32, [_vp, _vp]),
        "nph_gpu_mlp_predict": (ctypes.c_int32, [_vp, _vp, ctypes.c_uint64, _vp]),
        "nph_gpu_mlp_gradients": (ctypes.c_int32, [_vp, _vp, _vp, ctypes.c_uint64, _vp,
                                                   P(ctypes.c_float)]),
        "nph_gpu_mlp_train": (ctypes.c_int32, [_vp, _vp, _vp, ctypes.c_uint64, _u32, _u32,
                                               ctypes.c_float, ctypes.c_uint64,
                                               P(ctypes.c_float)]),
        "nph_gpu_mlp_time_kernels": (ctypes.c_int32, [_vp, ctypes.c_uint64, _u32, P(ctypes.c_float),
                                                      P(ctypes.c_float)]),
        "nph_gpu_world_features": (ctypes.c_int32, [_vp, P(abi.WorldParams), ctypes.c_float, _vp,
                                                    _vp, _vp, ctypes.c_uint64]),
        "nph_gpu_solver_set_warm_start_model": (ctypes.c_int32, [_vp, _vp]),
        "nph_gpu_world_update_contacts": (ctypes.c_int32, [_vp, _vp, _u32]),
        "nph_gpu_world_converge": (ctypes.c_int32, [_vp, P(abi.WorldParams), ctypes.c_float,
                                                    _u32, ctypes.c_float, _u32, ctypes.c_float,
                                                    _vp, _vp, P(abi.ConvergeStats)]),
        "nph_gpu_collide": (ctypes.c_int32, [_vp, _vp, _vp, _vp, _vp, _u32, _vp]),
        "nph_gpu_collide_release": (None, []),
        "nph_gpu_world_hit_events": (ctypes.c_int32, [_vp, ctypes.c_float, _vp, _u32, P(_u32)]),
        "nph_gpu_batch_hit_events": (ctypes.c_int32, [_vp, ctypes.c_float, _vp, _u32, P(_u32)]),
        "nph_gpu_world_sleep_decision": (ctypes.c_int32, [_vp, _vp, _u32, _vp, ctypes.c_float, _vp, _vp,
                                                          _vp]),
        "nph_gpu_collide_async": (ctypes.c_int32, [_vp, _vp, _vp, _vp, _vp, _u32, _vp, _vp, _vp,
                                                   ctypes.c_uint64, _vp]),
        "nph_gpu_collide_workspace_bytes": (ctypes.c_uint64, [_u32]),
        "nph_gpu_broad_phase": (ctypes.c_int32, [_vp, _vp, _vp, _u32, ctypes.c_float, _vp, _vp, _u32,
                                                 P(_u32)]),
        "nph_gpu_warm_start_contacts": (ctypes.c_int32, [_vp, _vp, _u32, _vp]),
        "nph_gpu_batch_create": (ctypes.c_int32, [P(abi.SolverDesc), P(_vp)]),
        "nph_gpu_batch_destroy": (None, [_vp]),
        "nph_gpu_batch_stream": (_vp, [_vp]),
        "nph_gpu_batch_upload": (ctypes.c_int32, [_vp, P(abi.WorldView), _u32]),
        "nph_gpu_batch_step_async": (ctypes.c_int32, [_vp, P(abi.WorldParams), ctypes.c_float,
                                                      _u32]),
        "nph_gpu_batch_download": (ctypes.c_int32, [_vp, P(abi.WorldView), _u32]),
        "nph_gpu_phys_solve_worlds": (ctypes.c_int32, [_vp, P(abi.WorldParams), ctypes.c_float,
                                                       P(abi.WorldView), _u32]),
        "nph_gpu_batch_set_config": (ctypes.c_int32, [_vp, P(abi.BatchTuning)]),
        "nph_gpu_batch_set_pipeline": (ctypes.c_int32, [_vp, _u32]),
        "nph_gpu_batch_config_count": (_u32, []),
        "nph_gpu_batch_autotune": (ctypes.c_int32, [_vp, P(abi.WorldParams), ctypes.c_float,
                                                    _u32, P(abi.BatchTuning)]),
        "nph_gpu_batch_info": (ctypes.c_int32, [_vp, P(abi.BatchInfo)]),
        "nph_gpu_pass_config_count": (_u32, []),
        "nph_gpu_solver_autotune": (ctypes.c_int32, [_vp, P(abi.WorldParams), ctypes.c_float,
                                                     _u32, P(_u32)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _check(code: int, what: str):
    if code != abi.OK:
        raise SolverError(code, what)


class Solver:
    """One device solver (NphGpuSolver): owns its device buffers and stream."""

    def __init__(self, device: int = 0, stream: int | None = None, use_graph: bool = True,
                 body_capacity: int = 0, contact_capacity: int = 0, joint_capacity: int = 0):
        L = lib()
        self._m = 0  # manifolds of the world the device holds
        d = abi.SolverDesc()
        d.device = device
        d.stream = stream
        d.use_graph = 1 if use_graph else 0
        d.body_capacity = body_capacity
        d.contact_capacity = contact_capacity
        d.joint_capacity = joint_capacity
        h = _vp()
        _check(L.nph_gpu_solver_create(ctypes.byref(d), ctypes.byref(h)), "nph_gpu_solver_create")
        self._h = h
        self.L = L

    def close(self):
        if getattr(self, "_h", None):
            self.L.nph_gpu_solver_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self) -> int:
        return int(self.L.nph_gpu_solver_stream(self._h) or 0)

    def phys_solve(self, view: abi.View, params: abi.WorldParams, dt: float) -> None:
        """The drop-in for phys_solve: solves `view` in place."""
        cv = view.c_view()
        _check(self.L.nph_gpu_phys_solve(self._h, ctypes.byref(params), dt, ctypes.byref(cv)),
               "nph_gpu_phys_solve")
        self._m = len(view.contacts)

    def phys_solve_code(self, view: abi.View, params: abi.WorldParams, dt: float) -> int:
        cv = view.c_view()
        code = int(self.L.nph_gpu_phys_solve(self._h, ctypes.byref(params), dt, ctypes.byref(cv)))
        if code == abi.OK:
            self._m = len(view.contacts)
        return code

    def upload(self, view: abi.View) -> None:
        cv = view.c_view()
        _check(self.L.nph_gpu_world_upload(self._h, ctypes.byref(cv)), "nph_gpu_world_upload")
        self._m = len(view.contacts)

    def step_async(self, params: abi.WorldParams, dt: float, steps: int = 1) -> None:
        _check(self.L.nph_gpu_world_step_async(self._h, ctypes.byref(params), dt, steps),
               "nph_gpu_world_step_async")

    def download(self, view: abi.View) -> None:
        cv = view.c_view()
        _check(self.L.nph_gpu_world_download(self._h, ctypes.byref(cv)), "nph_gpu_world_download")

    def synchronize(self) -> None:
        _check(self.L.nph_gpu_solver_synchronize(self._h), "nph_gpu_solver_synchronize")

    def phys_solve_packed(self, packed: abi.Packed, params: abi.WorldParams, dt: float) -> None:
        """nph_gpu_phys_solve_packed: the packed inputs in, the packed outputs filled."""
        cin, cout = packed.c_input(), packed.c_output()
        _check(self.L.nph_gpu_phys_solve_packed(self._h, ctypes.byref(params), dt, ctypes.byref(cin),
                                                ctypes.byref(cout)), "nph_gpu_phys_solve_packed")

    def set_memory_limit(self, nbytes: int) -> None:
        """A budget for the record and row arrays (0: none); growth beyond it fails with
        OUT_OF_MEMORY before anything is touched."""
        _check(self.L.nph_gpu_solver_set_memory_limit(self._h, int(nbytes)),
               "nph_gpu_solver_set_memory_limit")

    def memory(self) -> int:
        """Bytes the record and row arrays hold now."""
        return int(self.L.nph_gpu_solver_memory(self._h))

    def set_wait_injection(self, extra: int) -> None:
        """Test hook: the dependency-driven passes' waits ask for `extra` more finished
        constraints than will come, so they give up (0: off)."""
        _check(self.L.nph_gpu_solver_set_wait_injection(self._h, int(extra)),
               "nph_gpu_solver_set_wait_injection")

    def stats(self) -> abi.StepStats:
        st = abi.StepStats()
        _check(self.L.nph_gpu_solver_stats(self._h, ctypes.byref(st)), "nph_gpu_solver_stats")
        return st

    def profile_step(self, params: abi.WorldParams, dt: float) -> list[dict]:
        """One resident step with every launch timed (CUDA events), per kind of kernel."""
        arr = (abi.KernelTime * 32)()
        n = _u32()
        _check(self.L.nph_gpu_world_profile_step(self._h, ctypes.byref(params), dt, arr, 32,
                                                 ctypes.byref(n)), "nph_gpu_world_profile_step")
        return [{"name": arr[i].name.decode(), "launches": arr[i].launches,
                 "units": arr[i].units, "total_ms": arr[i].total_ms,
                 "algorithmic_bytes": arr[i].algorithmic_bytes} for i in range(n.value)]

    def pass_config_count(self) -> int:
        return int(self.L.nph_gpu_pass_config_count())

    def set_pass_config(self, pass_kind: int, config: int) -> None:
        _check(self.L.nph_gpu_solver_set_pass_config(self._h, pass_kind, config),
               "nph_gpu_solver_set_pass_config")

    def sleep_decision(self, island_of: np.ndarray, removed: np.ndarray, time_to_sleep: float):
        """nph_gpu_world_sleep_decision for the uploaded world: (islands that sleep as a bool
        array, the island to split or None, kinematic bodies that sleep as a bool array)."""
        island_of = np.ascontiguousarray(island_of, np.uint32)
        removed = np.ascontiguousarray(removed, np.uint32)
        sleep = np.zeros(max(len(removed), 1), np.uint8)
        kin = np.zeros(max(len(island_of), 1), np.uint8)
        split = _u32()
        _check(self.L.nph_gpu_world_sleep_decision(self._h, island_of.ctypes.data, len(removed),
                                                   removed.ctypes.data, time_to_sleep, sleep.ctypes.data,
                                                   ctypes.byref(split), kin.ctypes.data),
               "nph_gpu_world_sleep_decision")
        k = int(split.value)
        return sleep[:len(removed)] != 0, (None if k == abi.NULL else k), kin[:len(island_of)] != 0

    def hit_events(self, threshold: float = 1.0, capacity: int | None = None) -> np.ndarray:
        """nph_gpu_world_hit_events after a step: the hits in the view's order (the contact's
        index, its point of fastest approach, the approach speed)."""
        count = _u32()
        if capacity is None:  # the count first, then every event
            _check(self.L.nph_gpu_world_hit_events(self._h, threshold, None, 0, ctypes.byref(count)),
                   "nph_gpu_world_hit_events")
            capacity = int(count.value)
        out = np.zeros(max(capacity, 1), abi.HIT_EVENT_DTYPE)
        _check(self.L.nph_gpu_world_hit_events(self._h, threshold, out.ctypes.data, capacity,
                                               ctypes.byref(count)), "nph_gpu_world_hit_events")
        return out[:min(int(count.value), capacity)]

    def update_contacts(self, fresh: np.ndarray) -> None:
        """This step's manifolds (one per uploaded contact, same order, impulses zero),
        warm-started on the device from the records the last step stored."""
        fresh = np.ascontiguousarray(fresh, abi.CONTACT_DTYPE)
        _check(self.L.nph_gpu_world_update_contacts(self._h, fresh.ctypes.data, len(fresh)),
               "nph_gpu_world_update_contacts")

    def features(self, params: abi.WorldParams, dt: float):
        """Features (4m x 16), impulse scales and kinds of every point slot of the uploaded
        world at the step's start."""
        slots = 4 * int(self._m)
        f = np.zeros((slots, abi.MLP_INPUTS), np.float32)
        sc = np.zeros(slots, np.float32)
        kind = np.zeros(slots, np.uint32)
        _check(self.L.nph_gpu_world_features(self._h, ctypes.byref(params), dt, f.ctypes.data,
                                             sc.ctypes.data, kind.ctypes.data, slots),
               "nph_gpu_world_features")
        return f, sc, kind

    def set_warm_start_model(self, mlp) -> None:
        _check(self.L.nph_gpu_solver_set_warm_start_model(self._h, None if mlp is None
                                                          else mlp.handle),
               "nph_gpu_solver_set_warm_start_model")

    def converge(self, params: abi.WorldParams, dt: float, learned=False,
                 tolerance: float = 1e-4, max_passes: int = 2000,
                 reference_residual: float = 0.0, impulses: bool = False) -> dict:
        """The residual-driven mode on the uploaded world (nph_gpu_world_converge). `learned`:
        False/True (the plain or the network's start) or an abi.START_* value (START_GATED: the
        network's start with the plain start as its fallback)."""
        res = np.zeros(max_passes + 1, np.float32)
        imp = np.zeros(12 * int(self._m), np.float32) if impulses else None
        st = abi.ConvergeStats()
        _check(self.L.nph_gpu_world_converge(self._h, ctypes.byref(params), dt, int(learned),
                                             tolerance, max_passes, reference_residual,
                                             res.ctypes.data,
                                             None if imp is None else imp.ctypes.data,
                                             ctypes.byref(st)), "nph_gpu_world_converge")
        out = {k: getattr(st, k) for k, _ in abi.ConvergeStats._fields_}
        out["residuals"] = res[: st.passes + 1].copy()
        if imp is not None:
            out["impulses"] = imp.reshape(-1, 4, 3)
        return out

    def autotune(self, params: abi.WorldParams, dt: float, rounds: int = 1) -> list[int]:
        """Picks the fastest launch configuration per pass kind on the uploaded world."""
        chosen = (_u32 * 4)()
        _check(self.L.nph_gpu_solver_autotune(self._h, ctypes.byref(params), dt, rounds, chosen),
               "nph_gpu_solver_autotune")
        return list(chosen)

    def graph_color(self, body_a, body_b, dynamic_bits, body_slots: int):
        """Device colouring of constraints in insertion order (graph_pick_color)."""
        a = np.ascontiguousarray(body_a, np.uint32)
        b = np.ascontiguousarray(body_b, np.uint32)
        d = np.ascontiguousarray(dynamic_bits, np.uint8)
        color = np.zeros(len(a), np.uint32)
        slot = np.zeros(len(a), np.uint32)
        _check(self.L.nph_gpu_graph_color(self._h, a.ctypes.data, b.ctypes.data, d.ctypes.data,
                                          len(a), body_slots, color.ctypes.data,
                                          slot.ctypes.data), "nph_gpu_graph_color")
        return color, slot


class Mlp:
    """The learned warm start's network (NphGpuMlp): BF16 weights on the tensor cores, FP32
    master weights trained with Adam by the library's own kernels."""

    def __init__(self, device: int = 0, seed: int = 0):
        L = lib()
        h = _vp()
        _check(L.nph_gpu_mlp_create(device, seed, ctypes.byref(h)), "nph_gpu_mlp_create")
        self._h = h
        self.L = L

    def close(self):
        if getattr(self, "_h", None):
            self.L.nph_gpu_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def get_weights(self) -> np.ndarray:
        w = np.zeros(abi.MLP_PARAMS, np.float32)
        _check(self.L.nph_gpu_mlp_get_weights(self._h, w.ctypes.data), "nph_gpu_mlp_get_weights")
        return w

    def set_weights(self, w: np.ndarray) -> None:
        w = np.ascontiguousarray(w, np.float32)
        assert w.shape == (abi.MLP_PARAMS,)
        _check(self.L.nph_gpu_mlp_set_weights(self._h, w.ctypes.data), "nph_gpu_mlp_set_weights")

    def predict(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32).reshape(-1, abi.MLP_INPUTS)
        y = np.zeros((len(x), abi.MLP_OUTPUTS), np.float32)
        _check(self.L.nph_gpu_mlp_predict(self._h, x.ctypes.data, len(x), y.ctypes.data),
               "nph_gpu_mlp_predict")
        return y

    def gradients(self, x: np.ndarray, t: np.ndarray) -> tuple[np.ndarray, float]:
        x = np.ascontiguousarray(x, np.float32).reshape(-1, abi.MLP_INPUTS)
        t = np.ascontiguousarray(t, np.float32).reshape(-1, abi.MLP_OUTPUTS)
        g = np.zeros(abi.MLP_PARAMS, np.float32)
        loss = ctypes.c_float()
        _check(self.L.nph_gpu_mlp_gradients(self._h, x.ctypes.data, t.ctypes.data, len(x),
                                            g.ctypes.data, ctypes.byref(loss)),
               "nph_gpu_mlp_gradients")
        return g, float(loss.value)

    def time_kernels(self, count: int, reps: int = 5) -> dict:
        """nph_gpu_mlp_time_kernels: device milliseconds of one forward and one gradient
        launch over `count` device-resident synthetic rows."""
        f, g = ctypes.c_float(), ctypes.c_float()
        _check(self.L.nph_gpu_mlp_time_kernels(self._h, count, reps, ctypes.byref(f), ctypes.byref(g)),
               "nph_gpu_mlp_time_kernels")
        return {"forward_ms": float(f.value), "gradients_ms": float(g.value)}

    def train(self, x: np.ndarray, t: np.ndarray, epochs: int, batch: int, lr: float,
              seed: int = 0) -> float:
        x = np.ascontiguousarray(x, np.float32).reshape(-1, abi.MLP_INPUTS)
        t = np.ascontiguousarray(t, np.float32).reshape(-1, abi.MLP_OUTPUTS)
        loss = ctypes.c_float()
        _check(self.L.nph_gpu_mlp_train(self._h, x.ctypes.data, t.ctypes.data, len(x), epochs,
                                        batch, lr, seed, ctypes.byref(loss)), "nph_gpu_mlp_train")
        return float(loss.value)


class Batch:
    """Many independent worlds stepped in one persistent launch (NphGpuBatch)."""

    def __init__(self, device: int = 0, use_graph: bool = True):
        L = lib()
        d = abi.SolverDesc()
        d.device = device
        d.use_graph = 1 if use_graph else 0
        h = _vp()
        _check(L.nph_gpu_batch_create(ctypes.byref(d), ctypes.byref(h)), "nph_gpu_batch_create")
        self._h = h
        self.L = L
        self._views = None

    def close(self):
        if getattr(self, "_h", None):
            self.L.nph_gpu_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self) -> int:
        return int(self.L.nph_gpu_batch_stream(self._h) or 0)

    @staticmethod
    def _c_views(views):
        # The pointer keeps the array alive (numpy's data_as holds a reference to it).
        return abi.views_array(views).ctypes.data_as(ctypes.POINTER(abi.WorldView))

    def upload(self, views: list) -> None:
        self._views = views
        arr = self._c_views(views)
        _check(self.L.nph_gpu_batch_upload(self._h, arr, len(views)), "nph_gpu_batch_upload")

    def step_async(self, params: abi.WorldParams, dt: float, steps: int = 1) -> None:
        _check(self.L.nph_gpu_batch_step_async(self._h, ctypes.byref(params), dt, steps),
               "nph_gpu_batch_step_async")

    def download(self, views: list) -> None:
        arr = self._c_views(views)
        _check(self.L.nph_gpu_batch_download(self._h, arr, len(views)), "nph_gpu_batch_download")

    def phys_solve_worlds(self, views: list, params: abi.WorldParams, dt: float) -> None:
        arr = self._c_views(views)
        _check(self.L.nph_gpu_phys_solve_worlds(self._h, ctypes.byref(params), dt, arr,
                                                len(views)), "nph_gpu_phys_solve_worlds")

    def phys_solve_worlds_code(self, views: list, params: abi.WorldParams, dt: float) -> int:
        arr = self._c_views(views)
        return int(self.L.nph_gpu_phys_solve_worlds(self._h, ctypes.byref(params), dt, arr,
                                                    len(views)))

    def set_config(self, config: int = 3, shared_velocities: int = abi.BATCH_SHARED_SMALL,
                   items_per_thread: int = 2, packing: int = abi.BATCH_PERSISTENT) -> None:
        """Packing (abi.BATCH_PERSISTENT or abi.BATCH_MERGED); for the persistent packing the
        launch shape, shared-memory mode for velocities (abi.BATCH_SHARED_*) and the
        constraints a thread takes per colour when sizing a world's team (0: every world on a
        whole block)."""
        t = abi.BatchTuning()
        t.config = config
        t.shared_velocities = int(shared_velocities)
        t.items_per_thread = items_per_thread
        t.packing = packing
        _check(self.L.nph_gpu_batch_set_config(self._h, ctypes.byref(t)),
               "nph_gpu_batch_set_config")

    def hit_events(self, threshold: float = 1.0) -> np.ndarray:
        """nph_gpu_batch_hit_events after a step: every world's hits, world by world (`world`
        its place in the batch, `contact` the manifold's index in its view)."""
        count = _u32()
        _check(self.L.nph_gpu_batch_hit_events(self._h, threshold, None, 0, ctypes.byref(count)),
               "nph_gpu_batch_hit_events")
        cap = int(count.value)
        out = np.zeros(max(cap, 1), abi.HIT_EVENT_DTYPE)
        _check(self.L.nph_gpu_batch_hit_events(self._h, threshold, out.ctypes.data, cap, ctypes.byref(count)),
               "nph_gpu_batch_hit_events")
        return out[:min(int(count.value), cap)]

    def set_merged_pass_configs(self, configs) -> None:
        """The merged packing's pass configuration per pass kind (warm start, solve, relax,
        restitution), as Solver.set_pass_config."""
        for kind, config in enumerate(configs):
            _check(self.L.nph_gpu_batch_set_pass_config(self._h, kind, int(config)),
                   "nph_gpu_batch_set_pass_config")

    def set_pipeline(self, parts: int) -> None:
        """phys_solve_worlds in `parts` consecutive runs of worlds, each on its own stream, so
        that one part's results come back while later parts' records go up (1: unsplit)."""
        _check(self.L.nph_gpu_batch_set_pipeline(self._h, parts), "nph_gpu_batch_set_pipeline")

    def config_count(self) -> int:
        return int(self.L.nph_gpu_batch_config_count())

    def autotune(self, params: abi.WorldParams, dt: float, rounds: int = 1) -> dict:
        t = abi.BatchTuning()
        _check(self.L.nph_gpu_batch_autotune(self._h, ctypes.byref(params), dt, rounds,
                                             ctypes.byref(t)), "nph_gpu_batch_autotune")
        return {"config": t.config, "threads": t.threads,
                "shared_velocities": t.shared_velocities, "items_per_thread": t.items_per_thread,
                "packing": t.packing,
                "ms_per_step": t.ms_per_step, "persistent_ms_per_step": t.persistent_ms_per_step,
                "merged_ms_per_step": t.merged_ms_per_step}

    def info(self) -> dict:
        i = abi.BatchInfo()
        _check(self.L.nph_gpu_batch_info(self._h, ctypes.byref(i)), "nph_gpu_batch_info")
        return {k: getattr(i, k) for k, _ in abi.BatchInfo._fields_}


def collide(a: np.ndarray, pose_a: np.ndarray, b: np.ndarray, pose_b: np.ndarray,
            speculative: np.ndarray) -> np.ndarray:
    """The narrow phase on the device for pairs of spheres, capsules and boxes (nph_gpu_collide)."""
    a = np.ascontiguousarray(a, abi.SHAPE_DTYPE)
    b = np.ascontiguousarray(b, abi.SHAPE_DTYPE)
    pa = np.ascontiguousarray(pose_a, abi.POSE_DTYPE)
    pb = np.ascontiguousarray(pose_b, abi.POSE_DTYPE)
    sp = np.ascontiguousarray(speculative, np.float32)
    n = len(a)
    assert len(b) == len(pa) == len(pb) == len(sp) == n
    out = np.zeros(n, abi.MANIFOLD_DTYPE)
    _check(lib().nph_gpu_collide(a.ctypes.data, pa.ctypes.data, b.ctypes.data, pb.ctypes.data,
                                 sp.ctypes.data, n, out.ctypes.data), "nph_gpu_collide")
    return out


def collide_host(a_ptr: int, pose_a_ptr: int, b_ptr: int, pose_b_ptr: int, speculative_ptr: int,
                 count: int, out_ptr: int) -> None:
    """nph_gpu_collide on host arrays given by address (page-locked arrays let its chunks'
    copies overlap); synchronous."""
    _check(lib().nph_gpu_collide(a_ptr, pose_a_ptr, b_ptr, pose_b_ptr, speculative_ptr, count,
                                 out_ptr), "nph_gpu_collide")


def collide_release() -> None:
    """Frees the device arrays nph_gpu_collide keeps between calls."""
    lib().nph_gpu_collide_release()


def collide_workspace_bytes(count: int) -> int:
    return int(lib().nph_gpu_collide_workspace_bytes(count))


def collide_async(a_ptr: int, pose_a_ptr: int, b_ptr: int, pose_b_ptr: int, speculative_ptr: int,
                  count: int, out_ptr: int, bad_pairs_ptr: int = 0, workspace_ptr: int = 0,
                  workspace_bytes: int = 0, stream: int = 0) -> None:
    """nph_gpu_collide_async on device arrays (raw device pointers), enqueued on `stream`; with a
    workspace the pairs are sorted by kind on the device first."""
    _check(lib().nph_gpu_collide_async(a_ptr, pose_a_ptr, b_ptr, pose_b_ptr, speculative_ptr, count,
                                       out_ptr, bad_pairs_ptr or None, workspace_ptr or None,
                                       workspace_bytes, stream or None), "nph_gpu_collide_async")


def version() -> str:
    return lib().nph_gpu_version().decode()


def broad_phase(lo: np.ndarray, hi: np.ndarray, group: np.ndarray, cell: float):
    """nph_gpu_broad_phase: (pair_a, pair_b) of the boxes whose bounds overlap, within groups."""
    L = lib()
    lo = np.ascontiguousarray(lo, np.float32)
    hi = np.ascontiguousarray(hi, np.float32)
    group = np.ascontiguousarray(group, np.uint32)
    cap = max(16, 8 * len(lo))
    while True:
        a = np.zeros(cap, np.uint32)
        b = np.zeros(cap, np.uint32)
        n = _u32()
        _check(L.nph_gpu_broad_phase(lo.ctypes.data, hi.ctypes.data, group.ctypes.data, len(lo),
                                     float(cell), a.ctypes.data, b.ctypes.data, cap, ctypes.byref(n)),
               "nph_gpu_broad_phase")
        if n.value <= cap:
            return a[: n.value], b[: n.value]
        cap = n.value


def warm_start_contacts(old: np.ndarray, fresh: np.ndarray) -> np.ndarray:
    """nph_gpu_warm_start_contacts over aligned record arrays."""
    old = np.ascontiguousarray(old, abi.CONTACT_DTYPE)
    fresh = np.ascontiguousarray(fresh, abi.CONTACT_DTYPE)
    assert len(old) == len(fresh)
    out = np.zeros_like(fresh)
    _check(lib().nph_gpu_warm_start_contacts(old.ctypes.data, fresh.ctypes.data, len(out),
                                             out.ctypes.data), "nph_gpu_warm_start_contacts")
    return out
