"""ctypes binding of the C ABI in include/rumd_b200.h.

This is the thinnest host layer over the native engine: it loads the in-tree
``librumd_b200.so`` and fails loudly when it is missing -- there is no CPU or
PyTorch fallback.  ``Engine`` below is a convenience wrapper with numpy I/O;
the RUMD class surface (Sample, Pot_LJ_12_6, IntegratorNVT) is in
``rumd_b200.rumd`` on top of the C++ classes.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "librumd_b200.so")

B2MD_OK, B2MD_ERR_ARG, B2MD_ERR_CUDA, B2MD_ERR_NOMEM, B2MD_ERR_STATE, B2MD_ERR_OVERFLOW = range(6)
CUTOFF = {"NS": 0, "SP": 1, "SF": 2}
# pair functions (which RUMD Pot_* class the parameter rows belong to)
POTENTIAL = {"LJ_12_6": 0, "LJ_12_6_smooth_2_4": 1, "IPL_n": 2}
# kernel variants (b2md_engine_set_variant)
VARIANT_FORCE_MODE, VARIANT_BUILD_LANES, VARIANT_BUILD_SMEM, VARIANT_WINDOW_CAP, VARIANT_SM_TILES = 0, 1, 2, 3, 4
VARIANT_WINDOW_LIST_ROWS, VARIANT_PERSISTENT, VARIANT_PERSISTENT_ACTIVE, VARIANT_GRAPH_BUILDS = 5, 6, 7, 8
VARIANT_SPLIT_SORT_TILES = 9
FORCE_STREAMED, FORCE_STAGED, FORCE_WINDOW = 0, 1, 2
FIELD = {"pos": 0, "vel": 1, "force": 2, "virial": 3, "images": 4, "stress": 5}
STAT_NAMES = ["pe", "virial", "ke", "xi", "ke2", "steps", "rebuilds", "steps_left", "overflow",
              "target_T", "max_nbrs", "actual_max_nbrs", "mean_nbrs", "window_tiles", "tiles"]
NSTAT = len(STAT_NAMES)
NB_METHOD = {"default": -1, "sort": 0, "n2": 1}
COUNTER_NAMES = ["graph_builds", "graphs_dropped_by_layout", "graphs_dropped_by_pool_growth",
                 "graphs_dropped_by_list_repair", "graphs_dropped_by_settings", "list_repairs", "layouts", "chunks"]
# per-replica fields of a chunk's snapshot (b2md_run_queued_wait)
CHUNK_FIELDS = ["active", "steps", "steps_left", "pe", "virial", "ke", "xi", "rebuilds", "overflow"]

EXPORTS = [
    "b2md_engine_create", "b2md_engine_destroy", "b2md_engine_set_launch", "b2md_engine_get_launch",
    "b2md_engine_memory", "b2md_engine_usage", "b2md_engine_counters", "b2md_replica_footprint", "b2md_run_queued_async",
    "b2md_run_queued_poll", "b2md_run_queued_wait",
    "b2md_engine_set_graph_mode", "b2md_engine_set_variant", "b2md_engine_get_variant", "b2md_replica_add", "b2md_replica_remove", "b2md_replica_get",
    "b2md_replica_read", "b2md_replica_set", "b2md_replica_set_potential", "b2md_replica_add_potential", "b2md_replica_set_integrator",
    "b2md_replica_set_xi", "b2md_replica_set_reset_interval", "b2md_replica_set_nb_method",
    "b2md_replica_stats", "b2md_replica_set_energy_log", "b2md_replica_energy_log", "b2md_replica_stress", "b2md_calc_f",
    "b2md_integrate", "b2md_zero_momentum", "b2md_run", "b2md_run_timed", "b2md_replica_queue_steps",
    "b2md_run_queued", "b2md_nbl_export", "b2md_sort_export", "b2md_cell_grid", "b2md_sync",
    "b2md_stream", "b2md_last_error", "b2md_version", "b2md_probe_dist2", "b2md_probe_cell",
    "b2md_probe_nvt", "b2md_measure_peaks",
    "b2md_forces_noalloc", "b2md_f64_create", "b2md_f64_destroy", "b2md_f64_set_state",
    "b2md_f64_set_integrator", "b2md_f64_set_xi", "b2md_f64_calc_f", "b2md_f64_run", "b2md_f64_get",
    "b2md_f64_stats",
]


class ReplicaDesc(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int), ("ntypes", ctypes.c_int), ("box", ctypes.c_float * 3),
        ("params", ctypes.POINTER(ctypes.c_float)), ("cutoff_method", ctypes.c_int),
        ("skin", ctypes.c_float), ("dt", ctypes.c_float), ("target_T", ctypes.c_double),
        ("tau", ctypes.c_double), ("dT_per_step", ctypes.c_double), ("xi", ctypes.c_double),
        ("thermostat_mask", ctypes.c_uint), ("reset_interval", ctypes.c_int),
        ("max_nbrs", ctypes.c_int), ("energy_interval", ctypes.c_int),
        ("energy_capacity", ctypes.c_int), ("potential", ctypes.c_int),
    ]


_lib = None


def lib():
    """Loads librumd_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m rumd_b200.build` (no CPU fallback exists)")
        L = ctypes.CDLL(LIB_PATH)
        P, i, ll, f, d, u = (ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_float,
                             ctypes.c_double, ctypes.c_uint)
        sig = {
            "b2md_engine_create": [i, ll, i, ll, i, i, ctypes.POINTER(P)],
            "b2md_engine_destroy": [P],
            "b2md_engine_set_launch": [P, i, i],
            "b2md_engine_get_launch": [P, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)],
            "b2md_engine_memory": [P, ctypes.POINTER(ll)],
            "b2md_engine_usage": [P, ctypes.POINTER(ll), ctypes.POINTER(ll)],
            "b2md_engine_counters": [P, P, i],
            "b2md_replica_footprint": [P, ctypes.POINTER(ReplicaDesc), ctypes.POINTER(ll)],
            "b2md_run_queued_async": [P, ll, ctypes.POINTER(ll)],
            "b2md_run_queued_poll": [P, ll, ctypes.POINTER(i)],
            "b2md_run_queued_wait": [P, ll, ctypes.POINTER(ll), P, i],
            "b2md_engine_set_graph_mode": [P, i],
            "b2md_engine_set_variant": [P, i, i],
            "b2md_engine_get_variant": [P, i, ctypes.POINTER(ctypes.c_int)],
            "b2md_replica_add": [P, ctypes.POINTER(ReplicaDesc), P, P, P, ctypes.POINTER(i)],
            "b2md_replica_remove": [P, i],
            "b2md_replica_get": [P, i, i, P],
            "b2md_replica_read": [P, i, P, P, P],
            "b2md_replica_set": [P, i, i, P],
            "b2md_replica_set_potential": [P, i, i, P, i, f, i],
            "b2md_replica_add_potential": [P, i, i, P, i, i],
            "b2md_replica_set_integrator": [P, i, f, d, d, d, u],
            "b2md_replica_set_xi": [P, i, d],
            "b2md_replica_set_reset_interval": [P, i, i],
            "b2md_replica_set_nb_method": [P, i, i],
            "b2md_replica_stats": [P, i, P],
            "b2md_replica_set_energy_log": [P, i, i, i],
            "b2md_replica_energy_log": [P, i, P, i, ctypes.POINTER(i)],
            "b2md_replica_stress": [P, i, i, P],
            "b2md_calc_f": [P, i],
            "b2md_integrate": [P],
            "b2md_zero_momentum": [P],
            "b2md_run": [P, ll],
            "b2md_run_timed": [P, ll, ctypes.POINTER(d), ctypes.POINTER(ll)],
            "b2md_replica_queue_steps": [P, i, ll],
            "b2md_run_queued": [P, ll, ctypes.POINTER(ll)],
            "b2md_nbl_export": [P, i, P, P, i],
            "b2md_sort_export": [P, i, P],
            "b2md_cell_grid": [P, i, P],
            "b2md_sync": [P],
            "b2md_probe_dist2": [P, P, P, i, P],
            "b2md_probe_cell": [P, i, f, i, P],
            "b2md_probe_nvt": [P, P, P, P, f, P, i, P, P],
            "b2md_measure_peaks": [i, ctypes.POINTER(d), ctypes.POINTER(d)],
            "b2md_forces_noalloc": [P, i, P, i, P, i, P, P, P],
            "b2md_f64_create": [i, i, i, P, P, i, d, i, ctypes.POINTER(P)],
            "b2md_f64_destroy": [P],
            "b2md_f64_set_state": [P, P, P, P],
            "b2md_f64_set_integrator": [P, d, d, d, i, i],
            "b2md_f64_set_xi": [P, d],
            "b2md_f64_calc_f": [P],
            "b2md_f64_run": [P, ll, P],
            "b2md_f64_get": [P, i, P],
            "b2md_f64_stats": [P, P],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int
        L.b2md_stream.argtypes = [P]
        L.b2md_stream.restype = P
        L.b2md_last_error.restype = ctypes.c_char_p
        L.b2md_version.restype = ctypes.c_char_p
        _lib = L
    return _lib


class B2MDError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[b2md error {code}] {msg}")
        self.code = code


def check(rc):
    if rc != B2MD_OK:
        msg = lib().b2md_last_error().decode(errors="replace")
        if rc == B2MD_ERR_ARG:
            raise ValueError(msg)
        raise B2MDError(rc, msg)


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def pack_pos4(pos, types):
    """float32 [n,4]: xyz and the type bit-cast into the fourth lane."""
    pos = np.asarray(pos)
    n = len(pos)
    out = np.zeros((n, 4), np.float32)
    out[:, :3] = pos[:, :3]
    out[:, 3] = np.asarray(types, np.int32).view(np.float32)
    return out


def pack_vel4(vel, masses_per_particle):
    vel = np.asarray(vel)
    out = np.zeros((len(vel), 4), np.float32)
    out[:, :3] = vel[:, :3]
    out[:, 3] = 1.0 / np.asarray(masses_per_particle, np.float32)
    return out


def _desc(n, box, params, ntypes, cutoff="SF", skin=0.3, dt=0.005, T=1.0, tau=0.2, thermostat=True, xi=0.0,
          reset_interval=100, max_nbrs=0, dT_per_step=0.0, energy_interval=0, energy_capacity=0,
          thermostat_mask=None, potential="LJ_12_6"):
    """b2md_replica_desc of a system (params: float32, kept alive by the caller)."""
    d = ReplicaDesc()
    d.n, d.ntypes = n, ntypes
    for k in range(3):
        d.box[k] = float(box[k])
    d.params = params.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    d.cutoff_method = CUTOFF[cutoff] if isinstance(cutoff, str) else int(cutoff)
    d.skin, d.dt = skin, dt
    d.target_T, d.tau, d.dT_per_step, d.xi = T, tau, dT_per_step, xi
    if thermostat_mask is None:
        thermostat_mask = 0xFFFFFFFF if thermostat else 0
    d.thermostat_mask = thermostat_mask
    d.reset_interval = reset_interval
    d.max_nbrs = max_nbrs
    d.energy_interval, d.energy_capacity = energy_interval, energy_capacity
    d.potential = POTENTIAL[potential] if isinstance(potential, str) else int(potential)
    return d


class Engine:
    """Owns one b2md_engine: any number of resident MD systems on one GPU."""

    def __init__(self, device=0, max_particles=0, max_replicas=1, max_list_entries=0, pb=64, tp=4):
        h = ctypes.c_void_p()
        check(lib().b2md_engine_create(device, max_particles, max_replicas, max_list_entries, pb, tp,
                                       ctypes.byref(h)))
        self._h = h
        self._cap = max(int(max_replicas), 1)
        self.pb, self.tp = self.launch()

    def close(self):
        if getattr(self, "_h", None):
            lib().b2md_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def set_launch(self, pb, tp):
        """Sets (pb, tp); RUMD's shapes are mapped onto the engine's (see launch())."""
        check(lib().b2md_engine_set_launch(self._h, pb, tp))
        self.pb, self.tp = self.launch()

    def launch(self):
        """The (pb, tp) in effect after the engine's mapping of the requested shape."""
        p, t = ctypes.c_int(0), ctypes.c_int(0)
        check(lib().b2md_engine_get_launch(self._h, ctypes.byref(p), ctypes.byref(t)))
        return p.value, t.value

    def set_graph_mode(self, conditional):
        check(lib().b2md_engine_set_graph_mode(self._h, int(bool(conditional))))

    def set_variant(self, which, value):
        """which: VARIANT_FORCE_MODE, VARIANT_BUILD_LANES, VARIANT_BUILD_SMEM or VARIANT_WINDOW_CAP."""
        check(lib().b2md_engine_set_variant(self._h, int(which), int(value)))

    def get_variant(self, which):
        v = ctypes.c_int()
        check(lib().b2md_engine_get_variant(self._h, int(which), ctypes.byref(v)))
        return v.value

    def memory(self):
        b = ctypes.c_longlong()
        check(lib().b2md_engine_memory(self._h, ctypes.byref(b)))
        return b.value

    def usage(self):
        """(bytes held by the active replicas, bytes allocated by the engine)."""
        u, r = ctypes.c_longlong(), ctypes.c_longlong()
        check(lib().b2md_engine_usage(self._h, ctypes.byref(u), ctypes.byref(r)))
        return u.value, r.value

    def counters(self):
        """The engine's host-side event counters (b2md_engine_counters) by name."""
        out = np.zeros(len(COUNTER_NAMES), np.int64)
        check(lib().b2md_engine_counters(self._h, _ptr(out), len(COUNTER_NAMES)))
        return dict(zip(COUNTER_NAMES, out.tolist()))

    def footprint(self, n, box, params, ntypes, **kw):
        """Device bytes a replica of n particles would hold (b2md_replica_footprint);
        keywords as for add()."""
        params = np.ascontiguousarray(params, np.float32)
        d = _desc(n, box, params, ntypes, **kw)
        b = ctypes.c_longlong()
        check(lib().b2md_replica_footprint(self._h, ctypes.byref(d), ctypes.byref(b)))
        return b.value

    def add(self, pos4, box, params, ntypes, vel4=None, im3=None, **kw):
        """Admits one system; keywords: cutoff, skin, dt, T, tau, thermostat, xi,
        reset_interval, max_nbrs, dT_per_step, energy_interval, energy_capacity,
        thermostat_mask, potential."""
        pos4 = np.ascontiguousarray(pos4, np.float32)
        params = np.ascontiguousarray(params, np.float32)
        d = _desc(len(pos4), box, params, ntypes, **kw)
        v = None if vel4 is None else np.ascontiguousarray(vel4, np.float32)
        im = None if im3 is None else np.ascontiguousarray(im3, np.int32)
        rid = ctypes.c_int()
        check(lib().b2md_replica_add(self._h, ctypes.byref(d), _ptr(pos4), _ptr(v), _ptr(im), ctypes.byref(rid)))
        self._cap = max(self._cap, rid.value + 1)
        return rid.value

    def remove(self, rid):
        check(lib().b2md_replica_remove(self._h, rid))

    def get(self, rid, field, n):
        if field == "images":
            out = np.zeros((n, 3), np.int32)
        else:
            out = np.zeros((n, 4), np.float32)
        check(lib().b2md_replica_get(self._h, rid, FIELD[field], _ptr(out)))
        return out

    def read(self, rid, n, pos=True, vel=True, images=True):
        """Positions, velocities and images in original order, one id read-back."""
        p = np.zeros((n, 4), np.float32) if pos else None
        v = np.zeros((n, 4), np.float32) if vel else None
        im = np.zeros((n, 3), np.int32) if images else None
        check(lib().b2md_replica_read(self._h, rid, _ptr(p), _ptr(v), _ptr(im)))
        return p, v, im

    def set(self, rid, field, arr):
        dt = np.int32 if field == "images" else np.float32
        arr = np.ascontiguousarray(arr, dt)
        check(lib().b2md_replica_set(self._h, rid, FIELD[field], _ptr(arr)))

    def set_potential(self, rid, ntypes, params, cutoff, skin, potential="LJ_12_6"):
        params = np.ascontiguousarray(params, np.float32)
        c = CUTOFF[cutoff] if isinstance(cutoff, str) else int(cutoff)
        pk = POTENTIAL[potential] if isinstance(potential, str) else int(potential)
        check(lib().b2md_replica_set_potential(self._h, rid, ntypes, _ptr(params), c, skin, pk))

    def add_potential(self, rid, ntypes, params, cutoff, potential="LJ_12_6"):
        """A second pair potential whose forces and energies add to the first's."""
        params = np.ascontiguousarray(params, np.float32)
        c = CUTOFF[cutoff] if isinstance(cutoff, str) else int(cutoff)
        pk = POTENTIAL[potential] if isinstance(potential, str) else int(potential)
        check(lib().b2md_replica_add_potential(self._h, rid, ntypes, _ptr(params), c, pk))

    def set_integrator(self, rid, dt, T, tau, dT_per_step=0.0, thermostat_mask=0xFFFFFFFF):
        check(lib().b2md_replica_set_integrator(self._h, rid, dt, T, tau, dT_per_step, thermostat_mask))

    def set_xi(self, rid, xi):
        check(lib().b2md_replica_set_xi(self._h, rid, xi))

    def set_reset_interval(self, rid, k):
        check(lib().b2md_replica_set_reset_interval(self._h, rid, k))

    def set_nb_method(self, rid, method):
        check(lib().b2md_replica_set_nb_method(self._h, rid, NB_METHOD[method]))

    def stats(self, rid):
        out = np.zeros(NSTAT)
        check(lib().b2md_replica_stats(self._h, rid, _ptr(out)))
        return dict(zip(STAT_NAMES, out.tolist()))

    def set_energy_log(self, rid, interval, capacity):
        check(lib().b2md_replica_set_energy_log(self._h, rid, int(interval), int(capacity)))

    def energy_log(self, rid, cap=1 << 20):
        out = np.zeros((cap, 5))
        cnt = ctypes.c_int()
        check(lib().b2md_replica_energy_log(self._h, rid, _ptr(out), cap, ctypes.byref(cnt)))
        return out[: cnt.value]

    def stress(self, rid, include_kinetic=False):
        out = np.zeros(6)
        check(lib().b2md_replica_stress(self._h, rid, int(include_kinetic), _ptr(out)))
        return out

    def calc_f(self, stress=False):
        check(lib().b2md_calc_f(self._h, int(stress)))

    def integrate(self):
        check(lib().b2md_integrate(self._h))

    def zero_momentum(self):
        check(lib().b2md_zero_momentum(self._h))

    def run(self, nsteps):
        check(lib().b2md_run(self._h, int(nsteps)))

    def run_timed(self, nsteps):
        """Eager run with CUDA events around every fused step kernel: (kernel ms, launches)."""
        ms = ctypes.c_double()
        nl = ctypes.c_longlong()
        check(lib().b2md_run_timed(self._h, int(nsteps), ctypes.byref(ms), ctypes.byref(nl)))
        return ms.value, nl.value

    def stream(self):
        return lib().b2md_stream(self._h)

    def queue(self, rid, nsteps):
        check(lib().b2md_replica_queue_steps(self._h, rid, int(nsteps)))

    def run_queued(self, max_steps=0):
        n = ctypes.c_longlong()
        check(lib().b2md_run_queued(self._h, int(max_steps), ctypes.byref(n)))
        return n.value

    def run_queued_async(self, max_steps=0):
        """Launches a chunk of the queued work and returns its ticket at once."""
        t = ctypes.c_longlong()
        check(lib().b2md_run_queued_async(self._h, int(max_steps), ctypes.byref(t)))
        return t.value

    def poll(self, ticket):
        """True once the chunk has finished on the GPU (does not block)."""
        d = ctypes.c_int()
        check(lib().b2md_run_queued_poll(self._h, int(ticket), ctypes.byref(d)))
        return bool(d.value)

    def wait(self, ticket, cap=None):
        """Waits for a chunk: (steps it ran, [cap, len(CHUNK_FIELDS)] snapshot of
        every replica id's state at its end; rows of replicas not active at its
        launch have active 0 and steps_left -1)."""
        cap = self._cap if cap is None else cap
        out = np.zeros((cap, len(CHUNK_FIELDS)))
        n = ctypes.c_longlong()
        check(lib().b2md_run_queued_wait(self._h, int(ticket), ctypes.byref(n), _ptr(out), cap))
        return n.value, out

    def nbl(self, rid, n, max_nbrs):
        counts = np.zeros(n, np.uint32)
        nbl = np.zeros((n, max_nbrs), np.uint32)
        check(lib().b2md_nbl_export(self._h, rid, _ptr(counts), _ptr(nbl), max_nbrs))
        return counts, nbl

    def sort_index(self, rid, n):
        out = np.zeros(n, np.uint32)
        check(lib().b2md_sort_export(self._h, rid, _ptr(out)))
        return out

    def cell_grid(self, rid):
        out = np.zeros(3, np.int32)
        check(lib().b2md_cell_grid(self._h, rid, _ptr(out)))
        return out

    def sync(self):
        check(lib().b2md_sync(self._h))


def probe_dist2(a4, b4, box):
    a4 = np.ascontiguousarray(a4, np.float32)
    b4 = np.ascontiguousarray(b4, np.float32)
    box = np.ascontiguousarray(box, np.float32)
    out = np.zeros((len(a4), 2), np.float32)
    check(lib().b2md_probe_dist2(_ptr(a4), _ptr(b4), _ptr(box), len(a4), _ptr(out)))
    return out


def probe_cell(x, box, nc):
    x = np.ascontiguousarray(x, np.float32)
    out = np.zeros((len(x), 2), np.int32)
    check(lib().b2md_probe_cell(_ptr(x), len(x), float(box), int(nc), _ptr(out)))
    return out


def probe_nvt(r4, v4, f4, xi, dt, box):
    """(reference expressions, engine forms) of the leap-frog update: [n, 9] each."""
    r4, v4, f4 = (np.ascontiguousarray(x, np.float32) for x in (r4, v4, f4))
    xi = np.ascontiguousarray(xi, np.float32)
    box = np.ascontiguousarray(box, np.float32)
    ref = np.zeros((len(r4), 9), np.float32)
    eng = np.zeros((len(r4), 9), np.float32)
    check(lib().b2md_probe_nvt(_ptr(r4), _ptr(v4), _ptr(f4), _ptr(xi), float(dt), _ptr(box), len(r4), _ptr(ref),
                               _ptr(eng)))
    return ref, eng


def measure_peaks(trials=5):
    """(L2 read GB/s, FP32 FMA TFLOP/s) of the current device."""
    l2, fma = ctypes.c_double(0.0), ctypes.c_double(0.0)
    check(lib().b2md_measure_peaks(int(trials), ctypes.byref(l2), ctypes.byref(fma)))
    return l2.value, fma.value


F64_STAT_NAMES = ["pe", "virial", "ke", "ke2", "xi", "rebuilds", "steps"]


class F64Engine:
    """One system in the FP64 engine (b2md_f64_*): the accuracy oracle on the GPU.

    pos4 / vel4 as for Engine.add, but float64, with the type as a whole
    number in pos4[:, 3] (Engine's float32 pos4 with type bits is accepted
    too and converted)."""

    def __init__(self, pos4, box, params, ntypes, cutoff="SF", skin=0.3, dt=0.005, T=1.0, tau=0.2,
                 thermostat=True, reset_interval=100, vel4=None, im3=None, max_nbrs=0, device=0):
        pos4 = np.asarray(pos4)
        n = len(pos4)
        if pos4.dtype == np.float32:
            types = np.ascontiguousarray(pos4[:, 3]).view(np.int32).astype(np.float64)
            p = np.zeros((n, 4))
            p[:, :3] = pos4[:, :3]
            p[:, 3] = types
            pos4 = p
        pos4 = np.ascontiguousarray(pos4, np.float64)
        if vel4 is None:
            vel4 = np.zeros((n, 4))
            vel4[:, 3] = 1.0
        vel4 = np.ascontiguousarray(vel4, np.float64)
        im3 = None if im3 is None else np.ascontiguousarray(im3, np.int32)
        params = np.ascontiguousarray(params, np.float32)
        box3 = np.ascontiguousarray(np.broadcast_to(np.asarray(box, np.float64), (3,)))
        c = CUTOFF[cutoff] if isinstance(cutoff, str) else int(cutoff)
        self.n = n
        self._h = ctypes.c_void_p()
        check(lib().b2md_f64_create(int(device), n, int(ntypes), _ptr(box3), _ptr(params), c, float(skin),
                                    int(max_nbrs), ctypes.byref(self._h)))
        self.set_state(pos4, vel4, im3)
        self.set_integrator(dt, T, tau, thermostat, reset_interval)

    def close(self):
        if self._h:
            lib().b2md_f64_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, pos4, vel4, im3=None):
        pos4 = np.ascontiguousarray(pos4, np.float64)
        vel4 = np.ascontiguousarray(vel4, np.float64)
        im3 = None if im3 is None else np.ascontiguousarray(im3, np.int32)
        check(lib().b2md_f64_set_state(self._h, _ptr(pos4), _ptr(vel4), _ptr(im3)))

    def set_integrator(self, dt, T, tau, thermostat=True, reset_interval=100):
        check(lib().b2md_f64_set_integrator(self._h, float(dt), float(T), float(tau), int(bool(thermostat)),
                                            int(reset_interval)))

    def set_xi(self, xi):
        check(lib().b2md_f64_set_xi(self._h, float(xi)))

    def calc_f(self):
        check(lib().b2md_f64_calc_f(self._h))

    def run(self, nsteps, energies=False):
        """Runs nsteps; with energies=True returns [nsteps, 4] = pe, W, KE(t), xi."""
        en = np.zeros((int(nsteps), 4)) if energies else None
        check(lib().b2md_f64_run(self._h, int(nsteps), _ptr(en)))
        return en

    def get(self, field):
        """field: "pos", "vel", "force" ([n,4] float64) or "images" ([n,3] int32)."""
        if field == "images":
            out = np.zeros((self.n, 3), np.int32)
            check(lib().b2md_f64_get(self._h, 3, _ptr(out)))
            return out
        code = {"pos": 0, "vel": 1, "force": 2}[field]
        out = np.zeros((self.n, 4))
        check(lib().b2md_f64_get(self._h, code, _ptr(out)))
        return out

    def stats(self):
        out = np.zeros(len(F64_STAT_NAMES))
        check(lib().b2md_f64_stats(self._h, _ptr(out)))
        return dict(zip(F64_STAT_NAMES, out.tolist()))
