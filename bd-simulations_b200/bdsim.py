"""ctypes binding of libbd_b200.so (C ABI in include/bd_api.h).

Python mirror of the reference's run interface for tests and benchmarks:
`Run` wraps one bd_ctx with the RunDynamik routine names
(berechne_WCA11, berechne_kapkraefte, zeitschritt, ...), `Batch` wraps
bd_batch and `Server` wraps bd_server. Every call raises BdError on a
non-zero status; there is no fallback when the library or a GPU is missing.
"""
import ctypes as ct
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbd_b200.so")

NOISE_DISK, NOISE_GAUSS, NOISE_NONE = 0, 1, 2
FORCE_WCA, FORCE_KAP, FORCE_NOISE = 0, 1, 2
GRID_DENSITY, GRID_FX, GRID_FY = 0, 1, 2


class BdError(RuntimeError):
    def __init__(self, status, what):
        self.status = status
        super().__init__("%s failed: %s (%d)" % (what, _status_string(status), status))


class Params(ct.Structure):
    _fields_ = [
        ("N1", ct.c_int), ("N2", ct.c_int), ("L", ct.c_double),
        ("densGrid_Schema", ct.c_int), ("FFT_samples", ct.c_int),
        ("lambda_kapillar", ct.c_double), ("kapillar_vorfaktor", ct.c_double),
        ("T", ct.c_double), ("dt_max", ct.c_double), ("max_reisedistanz", ct.c_double),
        ("sigma11_22", ct.c_double), ("sigma11_12", ct.c_double), ("Gamma2_1", ct.c_double),
        ("eps22_11", ct.c_double), ("eps12_11", ct.c_double), ("f2_f1", ct.c_double),
        ("idgas_only", ct.c_int), ("noWCA", ct.c_int), ("noRNG", ct.c_int),
        ("quickInit", ct.c_int), ("restrictRadial", ct.c_int), ("debugmode", ct.c_int),
        ("krafttestmode", ct.c_int), ("maxPairWCA", ct.c_double),
        ("max_write_interval", ct.c_int), ("runs", ct.c_int), ("jobs", ct.c_int),
        ("maxThreads", ct.c_int), ("obs_dt", ct.c_double), ("obs_anzahl", ct.c_int),
        ("startpos_methode", ct.c_int), ("startpos_kreisradius", ct.c_double),
        ("noise_kind", ct.c_int), ("ngp_ref_compat", ct.c_int),
    ]


class Derived(ct.Structure):
    _fields_ = [("zweihoch1_6", ct.c_double), ("nachList_Zellen", ct.c_int),
                ("nachList_Breite", ct.c_double), ("densGrid_Breite", ct.c_double),
                ("densGrid_Zellen", ct.c_int), ("dq", ct.c_double), ("fixed_dt", ct.c_int)]


class TimestepInfo(ct.Structure):
    _fields_ = [("num_WCA_berechnet", ct.c_longlong), ("maxWCAx", ct.c_double), ("maxWCAy", ct.c_double),
                ("maxWCAtype", ct.c_int), ("maxWCAindex", ct.c_int), ("maxWCA_numWW1", ct.c_int),
                ("maxWCA_numWW2", ct.c_int), ("maxKapx", ct.c_double), ("maxKapy", ct.c_double),
                ("maxKaptype", ct.c_int), ("maxKapindex", ct.c_int), ("maxRNDx", ct.c_double),
                ("maxRNDy", ct.c_double), ("maxRNDtype", ct.c_int), ("maxRNDindex", ct.c_int),
                ("dt", ct.c_double), ("num_Zellwechsel1", ct.c_int), ("num_Zellwechsel2", ct.c_int),
                ("E_WCA", ct.c_double), ("virial_WCA", ct.c_double)]


class LokDensParams(ct.Structure):
    _fields_ = [("snapgrid_crude", ct.c_double), ("rhohist_bins", ct.c_int),
                ("rhohist_drho", ct.c_double), ("rho_thresh", ct.c_double * 3),
                ("drho_thresh", ct.c_double * 4)]


class ServeOpts(ct.Structure):
    _fields_ = [("device", ct.c_int), ("hbm_budget", ct.c_size_t), ("max_runs", ct.c_int),
                ("steps_per_tick", ct.c_int), ("snapshot_dir", ct.c_char_p)]


class ReqStatus(ct.Structure):
    _fields_ = [("state", ct.c_int), ("steps_done", ct.c_longlong),
                ("steps_total", ct.c_longlong), ("snapshots", ct.c_int),
                ("submit_s", ct.c_double), ("admit_s", ct.c_double), ("finish_s", ct.c_double),
                ("error", ct.c_int)]


class ServeStats(ct.Structure):
    _fields_ = [("completed", ct.c_longlong), ("particle_steps", ct.c_longlong),
                ("wall_s", ct.c_double), ("p50_latency_s", ct.c_double),
                ("p99_latency_s", ct.c_double), ("max_latency_s", ct.c_double),
                ("active", ct.c_int), ("queued", ct.c_int), ("hbm_in_use", ct.c_size_t),
                ("step_s", ct.c_double), ("host_s", ct.c_double), ("admit_s", ct.c_double),
                ("plan_s", ct.c_double), ("fetch_s", ct.c_double)]


class TuneResult(ct.Structure):
    _fields_ = [("dep_tiles_min", ct.c_int), ("fft_items_min", ct.c_int), ("dep_tile_max", ct.c_int),
                ("candidates", ct.c_int), ("default_ms", ct.c_double), ("best_ms", ct.c_double),
                ("particle_shape", ct.c_int), ("particle_default_ms", ct.c_double),
                ("particle_best_ms", ct.c_double)]


_lib = None

# every symbol include/bd_api.h declares
EXPORTS = [
    "bd_version", "bd_status_string", "bd_device_count", "bd_params_default",
    "bd_params_from_header", "bd_params_derived", "bd_create", "bd_destroy",
    "bd_init_positions", "bd_init_pos_aus_datei", "bd_set_positions", "bd_get_positions",
    "bd_WCA_init", "bd_kapkraefte_init", "bd_berechne_WCA11", "bd_berechne_WCA22",
    "bd_addiere_WCA12", "bd_berechne_kapkraefte", "bd_gridDensity_NGP", "bd_gridDensity_CIC",
    "bd_gridDensity_TSC", "bd_inv_gridDensity_NGP", "bd_inv_gridDensity_CIC",
    "bd_inv_gridDensity_TSC", "bd_berechne_zufallskraefte", "bd_optimaler_zeitschritt",
    "bd_refresh_erwNachbar", "bd_zeitschritt", "bd_zeitschritte", "bd_zeitschritte_bis_obs",
    "bd_get_forces", "bd_get_grid", "bd_get_list", "bd_get_step", "bd_set_step", "bd_get_time",
    "bd_sync", "bd_obs_init", "bd_schreibe_pos", "bd_write_pos_frame", "bd_init_positions_host",
    "bd_batch_create", "bd_batch_destroy", "bd_batch_step", "bd_batch_sync", "bd_batch_nruns",
    "bd_batch_get_positions", "bd_batch_set_positions", "bd_batch_set_positions_all",
    "bd_batch_get_positions_all", "bd_batch_get_time", "bd_run_footprint",
    "bd_serve_create", "bd_serve_destroy", "bd_serve_submit", "bd_serve_cancel",
    "bd_serve_poll", "bd_serve_tick", "bd_serve_result", "bd_serve_release",
    "bd_serve_snapshot", "bd_serve_stats_get", "bd_get_stream", "bd_batch_get_stream",
    "bd_launches_per_step", "bd_batch_launches_per_step", "bd_stage_times", "bd_batch_stage_times",
    "bd_set_positions_all", "bd_get_positions_all", "bd_gridDensity_noalloc", "bd_fused_phase_times",
    "bd_snapshot_save", "bd_snapshot_load", "bd_zeitschritt_info", "bd_korrelationsfunktion", "bd_ftrho",
    "bd_zeitschritt_debug", "bd_lokdens_params_default", "bd_lokdens_params_from_header", "bd_snapgrid_num", "bd_lokale_dichte",
    "bd_schreibe_lokale_dichte", "bd_batch_autotune", "bd_inject_barrier_timeout", "bd_batch_phase_times",
    "bd_batch_set_step_form",
]

STAGES = ["deposit", "fft_rows_fwd", "fft_cols_green", "fft_rows_inv", "particles",
          "scan", "scatter", "reserved7", "reserved8"]
# phases of the fused step (bd_fused_phase_times)
FUSED_PHASES = ["fft_rows_inv", "particles", "scan_next_fft_rows_fwd", "scatter_next_fft_cols_green"]


def lib():
    """Load the in-tree library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError("libbd_b200.so not built: run bd-simulations_b200/build.py")
        L = ct.CDLL(LIB_PATH)
        P, V, I, D = ct.POINTER, ct.c_void_p, ct.c_int, ct.c_double
        L.bd_version.restype = ct.c_char_p
        L.bd_status_string.restype = ct.c_char_p
        L.bd_status_string.argtypes = [I]
        sigs = {
            "bd_device_count": [P(I)],
            "bd_params_default": [P(Params)],
            "bd_params_from_header": [ct.c_char_p, P(Params)],
            "bd_params_derived": [P(Params), P(Derived)],
            "bd_create": [P(Params), ct.c_uint64, I, P(V)],
            "bd_destroy": [V],
            "bd_init_positions": [V, I],
            "bd_init_pos_aus_datei": [V, ct.c_char_p],
            "bd_set_positions": [V, I, V, V],
            "bd_get_positions": [V, I, V, V],
            "bd_optimaler_zeitschritt": [V, P(D)],
            "bd_zeitschritt": [V, D, P(D)],
            "bd_zeitschritte": [V, ct.c_longlong, P(D)],
            "bd_zeitschritte_bis_obs": [V, P(ct.c_longlong)],
            "bd_get_forces": [V, I, I, V],
            "bd_get_grid": [V, I, V],
            "bd_get_list": [V, I, I, I, V, I, P(I)],
            "bd_get_step": [V, P(ct.c_uint64)],
            "bd_set_step": [V, ct.c_uint64],
            "bd_get_time": [V, P(D)],
            "bd_obs_init": [V, I, ct.c_char_p],
            "bd_schreibe_pos": [V, I],
            "bd_write_pos_frame": [ct.c_char_p, I, D, I, V, V, D],
            "bd_init_positions_host": [P(Params), ct.c_uint64, I, V, V, V, V],
            "bd_batch_create": [V, V, I, I, P(V)],
            "bd_batch_destroy": [V],
            "bd_batch_step": [V, ct.c_longlong],
            "bd_batch_sync": [V],
            "bd_batch_nruns": [V, P(I)],
            "bd_batch_get_positions": [V, I, I, V, V],
            "bd_batch_set_positions": [V, I, I, V, V],
            "bd_batch_set_positions_all": [V, I, V, V, V, V],
            "bd_batch_get_positions_all": [V, I, V, V, V, V],
            "bd_batch_get_time": [V, I, P(D)],
            "bd_run_footprint": [P(Params), P(ct.c_size_t)],
            "bd_serve_create": [P(ServeOpts), P(V)],
            "bd_serve_destroy": [V],
            "bd_serve_submit": [V, P(Params), ct.c_uint64, ct.c_longlong, I, P(ct.c_longlong)],
            "bd_serve_cancel": [V, ct.c_longlong],
            "bd_serve_poll": [V, ct.c_longlong, P(ReqStatus)],
            "bd_serve_tick": [V, P(I)],
            "bd_serve_result": [V, ct.c_longlong, I, V, V],
            "bd_serve_release": [V, ct.c_longlong],
            "bd_serve_snapshot": [V, ct.c_longlong, I, P(ct.c_longlong), V, V],
            "bd_serve_stats_get": [V, P(ServeStats)],
            "bd_set_positions_all": [V, V, V, V, V],
            "bd_get_positions_all": [V, V, V, V, V],
            "bd_get_stream": [V, P(V)],
            "bd_batch_get_stream": [V, P(V)],
            "bd_launches_per_step": [V, P(I)],
            "bd_batch_launches_per_step": [V, P(I)],
            "bd_stage_times": [V, I, P(D), I],
            "bd_batch_stage_times": [V, I, P(D), I],
            "bd_batch_autotune": [V, I, P(TuneResult)],
            "bd_batch_set_step_form": [V, I, I],
            "bd_gridDensity_noalloc": [P(Params), I, V, V, V, V, V, V, V],
            "bd_fused_phase_times": [V, I, P(D), I],
            "bd_inject_barrier_timeout": [V, I, ct.c_uint],
            "bd_batch_phase_times": [V, I, P(D), I],
            "bd_snapshot_save": [V, ct.c_char_p],
            "bd_snapshot_load": [V, ct.c_char_p],
            "bd_zeitschritt_info": [V, P(TimestepInfo)],
            "bd_zeitschritt_debug": [V, D, P(TimestepInfo), P(D)],
            "bd_korrelationsfunktion": [V, I, D, I, V],
            "bd_ftrho": [V, I, I, D, V, V],
            "bd_lokdens_params_from_header": [ct.c_char_p, P(LokDensParams)],
            "bd_snapgrid_num": [P(Params), P(LokDensParams), P(I)],
            "bd_lokale_dichte": [V, P(LokDensParams), V, V, V, V],
            "bd_schreibe_lokale_dichte": [V, P(LokDensParams), ct.c_char_p, I],
        }
        for name in ["bd_sync", "bd_WCA_init", "bd_kapkraefte_init", "bd_berechne_WCA11",
                     "bd_berechne_WCA22", "bd_addiere_WCA12", "bd_berechne_kapkraefte",
                     "bd_gridDensity_NGP", "bd_gridDensity_CIC", "bd_gridDensity_TSC",
                     "bd_inv_gridDensity_NGP", "bd_inv_gridDensity_CIC", "bd_inv_gridDensity_TSC",
                     "bd_berechne_zufallskraefte", "bd_refresh_erwNachbar"]:
            sigs[name] = [V]
        for name, args in sigs.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = I
        L.bd_lokdens_params_default.argtypes = [P(LokDensParams)]
        L.bd_lokdens_params_default.restype = None
        _lib = L
    return _lib


def _status_string(s):
    try:
        return lib().bd_status_string(s).decode()
    except Exception:
        return "status"


def _ck(status, what):
    if status != 0:
        raise BdError(status, what)


def _ptr(a):
    return a.ctypes.data_as(ct.c_void_p) if a is not None else None


def default_params():
    p = Params()
    _ck(lib().bd_params_default(ct.byref(p)), "bd_params_default")
    return p


def params_from(d):
    """bd_params from a dict of reference parameter names over the defaults."""
    p = default_params()
    names = {n for n, _ in Params._fields_}
    for k, v in d.items():
        if k in names:
            typ = dict(Params._fields_)[k]
            setattr(p, k, int(v) if typ is ct.c_int else float(v))
    return p


def params_from_header(path):
    p = default_params()
    _ck(lib().bd_params_from_header(path.encode(), ct.byref(p)), "bd_params_from_header")
    return p


def lokdens_params(**kw):
    """Local-density parameters: the shipped values, then any of
    snapgrid_crude, rhohist_bins, rhohist_drho, rho_thresh (3),
    drho_thresh (4) given by name."""
    lp = LokDensParams()
    lib().bd_lokdens_params_default(ct.byref(lp))
    for k, v in kw.items():
        if k in ("rho_thresh", "drho_thresh"):
            arr = getattr(lp, k)
            if len(v) != len(arr):
                raise ValueError("%s takes %d values" % (k, len(arr)))
            for i, x in enumerate(v):
                arr[i] = float(x)
        elif k == "rhohist_bins":
            lp.rhohist_bins = int(v)
        elif k in ("snapgrid_crude", "rhohist_drho"):
            setattr(lp, k, float(v))
        else:
            raise KeyError(k)
    return lp


def lokdens_params_from_header(path):
    lp = lokdens_params()
    _ck(lib().bd_lokdens_params_from_header(path.encode(), ct.byref(lp)), "bd_lokdens_params_from_header")
    return lp


def derived(p):
    d = Derived()
    _ck(lib().bd_params_derived(ct.byref(p), ct.byref(d)), "bd_params_derived")
    return d


def device_count():
    n = ct.c_int(0)
    lib().bd_device_count(ct.byref(n))
    return n.value


def footprint(p):
    b = ct.c_size_t(0)
    _ck(lib().bd_run_footprint(ct.byref(p), ct.byref(b)), "bd_run_footprint")
    return b.value


def init_positions_host(p, seed, methode=1):
    n1, n2 = p.N1, p.N2
    g1 = np.zeros((n1, 2), np.int32)
    r1 = np.zeros((n1, 2))
    g2 = np.zeros((max(n2, 1), 2), np.int32)
    r2 = np.zeros((max(n2, 1), 2))
    _ck(lib().bd_init_positions_host(ct.byref(p), seed, methode, _ptr(g1), _ptr(r1), _ptr(g2), _ptr(r2)),
        "bd_init_positions_host")
    return {0: (g1, r1), 1: (g2[:n2], r2[:n2])}


def write_pos_frame(path, append, t, git, rel, B):
    git = np.ascontiguousarray(git, np.int32)
    rel = np.ascontiguousarray(rel, np.float64)
    _ck(lib().bd_write_pos_frame(path.encode(), int(append), float(t), len(git), _ptr(git), _ptr(rel), B),
        "bd_write_pos_frame")


class Run:
    """One run: RunZustand + RunDynamik routines through the C ABI."""

    def __init__(self, params, seed=0, device=0):
        self.p = params if isinstance(params, Params) else params_from(params)
        self.h = ct.c_void_p()
        _ck(lib().bd_create(ct.byref(self.p), seed, device, ct.byref(self.h)), "bd_create")
        self.N = (self.p.N1, self.p.N2)
        self.Z = self.p.FFT_samples
        d = derived(self.p)
        self.C, self.B = d.nachList_Zellen, d.nachList_Breite

    def close(self):
        if self.h:
            lib().bd_destroy(self.h)
            self.h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _call(self, name, *args):
        _ck(getattr(lib(), name)(self.h, *args), name)

    def init_positions(self, methode=1):
        self._call("bd_init_positions", methode)

    def set_positions(self, pos):
        for s in (0, 1):
            if self.N[s] == 0:
                continue
            g = np.ascontiguousarray(pos[s][0], np.int32)
            r = np.ascontiguousarray(pos[s][1], np.float64)
            self._call("bd_set_positions", s, _ptr(g), _ptr(r))

    def get_positions(self, out=None):
        """Both species in one device->host copy; `out` reuses host arrays."""
        if out is None:
            out = {s: (np.zeros((max(self.N[s], 1), 2), np.int32), np.zeros((max(self.N[s], 1), 2)))
                   for s in (0, 1)}
        self._call("bd_get_positions_all", _ptr(out[0][0]), _ptr(out[0][1]), _ptr(out[1][0]), _ptr(out[1][1]))
        return {s: (out[s][0][:self.N[s]], out[s][1][:self.N[s]]) for s in (0, 1)}

    def set_positions_all(self, pos):
        """Both species in one host->device copy."""
        a = [np.ascontiguousarray(pos[s][k], np.int32 if k == 0 else np.float64) for s in (0, 1) for k in (0, 1)]
        self._call("bd_set_positions_all", _ptr(a[0]), _ptr(a[1]), _ptr(a[2]) if self.N[1] else None,
                   _ptr(a[3]) if self.N[1] else None)

    # routines named as RunDynamik
    def WCA_init(self): self._call("bd_WCA_init")
    def berechne_WCA11(self): self._call("bd_berechne_WCA11")
    def berechne_WCA22(self): self._call("bd_berechne_WCA22")
    def addiere_WCA12(self): self._call("bd_addiere_WCA12")
    def berechne_kapkraefte(self): self._call("bd_berechne_kapkraefte")
    def gridDensity(self, scheme): self._call(["bd_gridDensity_NGP", "bd_gridDensity_CIC", "bd_gridDensity_TSC"][scheme])
    def inv_gridDensity(self, scheme): self._call(["bd_inv_gridDensity_NGP", "bd_inv_gridDensity_CIC", "bd_inv_gridDensity_TSC"][scheme])
    def berechne_zufallskraefte(self): self._call("bd_berechne_zufallskraefte")
    def refresh_erwNachbar(self): self._call("bd_refresh_erwNachbar")

    def optimaler_zeitschritt(self):
        dt = ct.c_double()
        self._call("bd_optimaler_zeitschritt", ct.byref(dt))
        return dt.value

    def zeitschritt(self, tmax=1.0):
        dt = ct.c_double()
        self._call("bd_zeitschritt", float(tmax), ct.byref(dt))
        return dt.value

    def zeitschritte(self, n):
        t = ct.c_double()
        self._call("bd_zeitschritte", int(n), ct.byref(t))
        return t.value

    def zeitschritte_bis_obs(self):
        n = ct.c_longlong()
        self._call("bd_zeitschritte_bis_obs", ct.byref(n))
        return n.value

    def forces(self):
        """Reference order: WCA11, WCA22, WCA12, capillary."""
        self.berechne_WCA11()
        self.berechne_WCA22()
        self.addiere_WCA12()
        self.berechne_kapkraefte()
        return self.get_forces()

    def get_forces(self):
        out = {}
        for kind, name in ((0, "wca"), (1, "kap"), (2, "noise")):
            for s in (0, 1):
                a = np.zeros((max(self.N[s], 1), 2))
                self._call("bd_get_forces", kind, s, _ptr(a))
                out[(name, s)] = a[:self.N[s]]
        return out

    def grid(self, which):
        a = np.zeros(self.Z * self.Z)
        self._call("bd_get_grid", which, _ptr(a))
        return a.reshape(self.Z, self.Z)

    def list(self, species, i, j):
        n = ct.c_int()
        self._call("bd_get_list", species, i, j, None, 0, ct.byref(n))
        a = np.zeros(max(n.value, 1), np.int32)
        self._call("bd_get_list", species, i, j, _ptr(a), n.value, ct.byref(n))
        return a[:n.value]

    def step_count(self):
        s = ct.c_uint64()
        self._call("bd_get_step", ct.byref(s))
        return s.value

    def set_step(self, s):
        self._call("bd_set_step", int(s))

    def time(self):
        t = ct.c_double()
        self._call("bd_get_time", ct.byref(t))
        return t.value

    def sync(self):
        self._call("bd_sync")

    def obs_init(self, run, directory):
        self._call("bd_obs_init", run, directory.encode())

    def schreibe_pos(self, nr):
        self._call("bd_schreibe_pos", nr)

    def stream(self):
        s = ct.c_void_p()
        self._call("bd_get_stream", ct.byref(s))
        return s.value

    def launches_per_step(self):
        n = ct.c_int()
        self._call("bd_launches_per_step", ct.byref(n))
        return n.value

    def stage_times(self, nsteps):
        ms = (ct.c_double * 9)()
        self._call("bd_stage_times", int(nsteps), ms, 9)
        return dict(zip(STAGES, list(ms)))

    def timestep_info(self):
        """TimestepInfo of the current positions and step (no move)."""
        info = TimestepInfo()
        self._call("bd_zeitschritt_info", ct.byref(info))
        return {n: getattr(info, n) for n, _ in TimestepInfo._fields_}

    def zeitschritt_debug(self, mrd):
        """One step of length optimaler_zeitschritt(mrd) with its TimestepInfo."""
        info = TimestepInfo()
        dt = ct.c_double()
        self._call("bd_zeitschritt_debug", float(mrd), ct.byref(info), ct.byref(dt))
        return {n: getattr(info, n) for n, _ in TimestepInfo._fields_}

    def korrelationsfunktion(self, which, dr, bins):
        g = np.zeros(bins)
        self._call("bd_korrelationsfunktion", int(which), float(dr), int(bins), _ptr(g))
        return g

    def ftrho(self, species, qbins, dq):
        re, im = np.zeros(qbins * qbins), np.zeros(qbins * qbins)
        self._call("bd_ftrho", int(species), int(qbins), float(dq), _ptr(re), _ptr(im))
        return (re + 1j * im).reshape(qbins, qbins)

    def lokale_dichte(self, lp=None):
        """Local densities of the resident state: (rho1, rho2) [n, n] (index
        [k, l], k along x), hist [4, bins] (rho1, rho2, rho1+rho2, rho1-rho2)
        and threshold counts over [7]."""
        lp = lp if lp is not None else lokdens_params()
        n = ct.c_int()
        _ck(lib().bd_snapgrid_num(ct.byref(self.p), ct.byref(lp), ct.byref(n)), "bd_snapgrid_num")
        n = n.value
        g1, g2 = np.zeros(n * n), np.zeros(n * n)
        hist = np.zeros((4, lp.rhohist_bins), np.int32)
        over = np.zeros(7, np.int32)
        self._call("bd_lokale_dichte", ct.byref(lp), _ptr(g1), _ptr(g2), _ptr(hist), _ptr(over))
        return g1.reshape(n, n), g2.reshape(n, n), hist, over

    def schreibe_lokale_dichte(self, directory, nr, lp=None):
        lp = lp if lp is not None else lokdens_params()
        self._call("bd_schreibe_lokale_dichte", ct.byref(lp), str(directory).encode(), int(nr))

    def snapshot_save(self, path):
        self._call("bd_snapshot_save", str(path).encode())

    def snapshot_load(self, path):
        self._call("bd_snapshot_load", str(path).encode())

    def fused_phase_times(self, nsteps):
        """Phase times of the fused step (ms per step), or None when this run
        steps with the stage kernels."""
        ms = (ct.c_double * len(FUSED_PHASES))()
        st = lib().bd_fused_phase_times(self.h, int(nsteps), ms, len(FUSED_PHASES))
        if st == -5:
            return None
        _ck(st, "bd_fused_phase_times")
        return dict(zip(FUSED_PHASES, list(ms)))


class Batch:
    """Many independent runs stepped together (bd_batch)."""

    def __init__(self, params_list, seeds, device=0):
        ps = [p if isinstance(p, Params) else params_from(p) for p in params_list]
        self.params = ps
        arr = (Params * len(ps))(*ps)
        sd = (ct.c_uint64 * len(ps))(*seeds)
        self.h = ct.c_void_p()
        _ck(lib().bd_batch_create(ct.cast(arr, ct.c_void_p), ct.cast(sd, ct.c_void_p), len(ps), device,
                                  ct.byref(self.h)), "bd_batch_create")

    def close(self):
        if self.h:
            lib().bd_batch_destroy(self.h)
            self.h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n):
        _ck(lib().bd_batch_step(self.h, int(n)), "bd_batch_step")

    def sync(self):
        _ck(lib().bd_batch_sync(self.h), "bd_batch_sync")

    def get_positions(self, run):
        """Both species of one run in one device->host copy."""
        p = self.params[run]
        out = {s: (np.zeros((max(n, 1), 2), np.int32), np.zeros((max(n, 1), 2)))
               for s, n in ((0, p.N1), (1, p.N2))}
        _ck(lib().bd_batch_get_positions_all(self.h, run, _ptr(out[0][0]), _ptr(out[0][1]), _ptr(out[1][0]),
                                             _ptr(out[1][1])), "bd_batch_get_positions_all")
        return {s: (out[s][0][:n], out[s][1][:n]) for s, n in ((0, p.N1), (1, p.N2))}

    def get_positions_species(self, run, species):
        """One species through bd_batch_get_positions."""
        n = (self.params[run].N1, self.params[run].N2)[species]
        g = np.zeros((max(n, 1), 2), np.int32)
        r = np.zeros((max(n, 1), 2))
        _ck(lib().bd_batch_get_positions(self.h, run, species, _ptr(g), _ptr(r)), "bd_batch_get_positions")
        return g[:n], r[:n]

    def set_positions(self, run, pos):
        """Both species of one run in one host->device copy and one sort."""
        p = self.params[run]
        a = [np.ascontiguousarray(pos[s][k], np.int32 if k == 0 else np.float64) for s in (0, 1) for k in (0, 1)]
        _ck(lib().bd_batch_set_positions_all(self.h, run, _ptr(a[0]), _ptr(a[1]), _ptr(a[2]) if p.N2 else None,
                                             _ptr(a[3]) if p.N2 else None), "bd_batch_set_positions_all")

    def set_positions_species(self, run, species, git, rel):
        """One species through bd_batch_set_positions (the other keeps its positions)."""
        g = np.ascontiguousarray(git, np.int32)
        r = np.ascontiguousarray(rel, np.float64)
        _ck(lib().bd_batch_set_positions(self.h, run, species, _ptr(g), _ptr(r)), "bd_batch_set_positions")

    def time(self, run):
        t = ct.c_double()
        _ck(lib().bd_batch_get_time(self.h, run, ct.byref(t)), "bd_batch_get_time")
        return t.value

    def stream(self):
        s = ct.c_void_p()
        _ck(lib().bd_batch_get_stream(self.h, ct.byref(s)), "bd_batch_get_stream")
        return s.value

    def launches_per_step(self):
        n = ct.c_int()
        _ck(lib().bd_batch_launches_per_step(self.h, ct.byref(n)), "bd_batch_launches_per_step")
        return n.value

    def stage_times(self, nsteps):
        ms = (ct.c_double * 9)()
        _ck(lib().bd_batch_stage_times(self.h, int(nsteps), ms, 9), "bd_batch_stage_times")
        return dict(zip(STAGES, list(ms)))

    def phase_times(self, nsteps):
        """Phase times (ms per step) of the pipelined stage step, or None when
        the batch steps with the classic stage kernels."""
        ms = (ct.c_double * len(FUSED_PHASES))()
        st = lib().bd_batch_phase_times(self.h, int(nsteps), ms, len(FUSED_PHASES))
        if st == -5:
            return None
        _ck(st, "bd_batch_phase_times")
        return dict(zip(FUSED_PHASES, list(ms)))

    def set_step_form(self, form, ctas_per_sm=0):
        """bd_batch_set_step_form: form 0 six launches per step (ctas_per_sm
        0), 1 two launches (the particle kernel and the cooperative tail at
        ctas_per_sm CTAs per SM)."""
        _ck(lib().bd_batch_set_step_form(self.h, int(form), int(ctas_per_sm)), "bd_batch_set_step_form")

    def autotune(self, reps=5):
        """bd_batch_autotune: times the candidate deposit-tile / transform-item
        plans and keeps the fastest; returns the TuneResult."""
        res = TuneResult()
        _ck(lib().bd_batch_autotune(self.h, int(reps), ct.byref(res)), "bd_batch_autotune")
        return res


class Server:
    """Continuous-batching request loop (bd_server)."""

    def __init__(self, device=0, hbm_budget=0, max_runs=0, steps_per_tick=100, snapshot_dir=None):
        self._dir = snapshot_dir.encode() if snapshot_dir else None
        o = ServeOpts(device, hbm_budget, max_runs, steps_per_tick, self._dir)
        self.h = ct.c_void_p()
        _ck(lib().bd_serve_create(ct.byref(o), ct.byref(self.h)), "bd_serve_create")
        self.params = {}

    def close(self):
        if self.h:
            lib().bd_serve_destroy(self.h)
            self.h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, params, seed, nsteps, snapshot_every=0):
        p = params if isinstance(params, Params) else params_from(params)
        rid = ct.c_longlong()
        _ck(lib().bd_serve_submit(self.h, ct.byref(p), seed, int(nsteps), int(snapshot_every), ct.byref(rid)),
            "bd_serve_submit")
        self.params[rid.value] = p
        return rid.value

    def cancel(self, rid):
        _ck(lib().bd_serve_cancel(self.h, rid), "bd_serve_cancel")

    def poll(self, rid):
        st = ReqStatus()
        _ck(lib().bd_serve_poll(self.h, rid, ct.byref(st)), "bd_serve_poll")
        return st

    def tick(self):
        a = ct.c_int()
        _ck(lib().bd_serve_tick(self.h, ct.byref(a)), "bd_serve_tick")
        return a.value

    def result(self, rid):
        p = self.params[rid]
        out = {}
        for s, n in ((0, p.N1), (1, p.N2)):
            g = np.zeros((max(n, 1), 2), np.int32)
            r = np.zeros((max(n, 1), 2))
            _ck(lib().bd_serve_result(self.h, rid, s, _ptr(g), _ptr(r)), "bd_serve_result")
            out[s] = (g[:n], r[:n])
        return out

    def release(self, rid):
        _ck(lib().bd_serve_release(self.h, rid), "bd_serve_release")

    def snapshot(self, rid, species=0):
        p = self.params[rid]
        n = p.N1 if species == 0 else p.N2
        g = np.zeros((max(n, 1), 2), np.int32)
        r = np.zeros((max(n, 1), 2))
        step = ct.c_longlong()
        _ck(lib().bd_serve_snapshot(self.h, rid, species, ct.byref(step), _ptr(g), _ptr(r)), "bd_serve_snapshot")
        return step.value, g[:n], r[:n]

    def stats(self):
        s = ServeStats()
        _ck(lib().bd_serve_stats_get(self.h, ct.byref(s)), "bd_serve_stats_get")
        return s
