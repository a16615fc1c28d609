"""ctypes binding of the C oracle (bd_oracle.c) and helpers around the
compiled reference checker. TEST INFRASTRUCTURE: imported only by tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline/reference leg.
"""
import ctypes as ct
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "liboracle.so")

NOISE_REF_STREAM, NOISE_INJECTED, NOISE_PHILOX_DISK, NOISE_PHILOX_GAUSS, NOISE_NONE = range(5)


class BdoParams(ct.Structure):
    _fields_ = [
        ("N1", ct.c_int), ("N2", ct.c_int), ("L", ct.c_double),
        ("densGrid_Schema", ct.c_int), ("FFT_samples", ct.c_int),
        ("lambda_kapillar", ct.c_double), ("kapillar_vorfaktor", ct.c_double),
        ("T", ct.c_double), ("dt_max", ct.c_double), ("max_reisedistanz", ct.c_double),
        ("sigma11_22", ct.c_double), ("sigma11_12", ct.c_double), ("Gamma2_1", ct.c_double),
        ("eps22_11", ct.c_double), ("eps12_11", ct.c_double), ("f2_f1", ct.c_double),
        ("idgas_only", ct.c_int), ("noWCA", ct.c_int), ("noRNG", ct.c_int),
        ("quickInit", ct.c_int), ("restrictRadial", ct.c_int),
        ("maxPairWCA", ct.c_double), ("obs_dt", ct.c_double),
        ("startpos_methode", ct.c_int), ("startpos_kreisradius", ct.c_double),
    ]


def build(force=False):
    """Compile liboracle.so (oracle + FFT shim). No FMA contraction, so the
    operation order written in bd_oracle.c is the one executed."""
    os.makedirs(BUILD, exist_ok=True)
    srcs = [os.path.join(HERE, "bd_oracle.c"), os.path.join(HERE, "fftw_shim", "fftw_shim.c")]
    hdrs = [os.path.join(HERE, "bd_oracle.h"), os.path.join(HERE, "fftw_shim", "fftw3.h")]
    if not force and os.path.exists(LIB):
        t = os.path.getmtime(LIB)
        if all(os.path.getmtime(s) < t for s in srcs + hdrs):
            return LIB
    cmd = ["gcc", "-O2", "-std=c99", "-D_GNU_SOURCE", "-ffp-contract=off", "-fPIC", "-shared",
           "-I" + HERE] + srcs + ["-lm", "-o", LIB]
    subprocess.run(cmd, check=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ct.CDLL(LIB)
        P = ct.POINTER
        L.bdo_create.restype = ct.c_void_p
        L.bdo_create.argtypes = [P(BdoParams), ct.c_uint64]
        L.bdo_destroy.argtypes = [ct.c_void_p]
        for n in ["bdo_WCA_init", "bdo_kapkraefte_init", "bdo_berechne_WCA11",
                  "bdo_berechne_WCA22", "bdo_addiere_WCA12", "bdo_berechne_kapkraefte",
                  "bdo_berechne_zufallskraefte", "bdo_refresh_erwNachbar"]:
            getattr(L, n).argtypes = [ct.c_void_p]
        L.bdo_gridDensity.argtypes = [ct.c_void_p, ct.c_int]
        L.bdo_inv_gridDensity.argtypes = [ct.c_void_p, ct.c_int]
        L.bdo_optimaler_zeitschritt.argtypes = [ct.c_void_p]
        L.bdo_optimaler_zeitschritt.restype = ct.c_double
        L.bdo_zeitschritt.argtypes = [ct.c_void_p, ct.c_double]
        L.bdo_zeitschritt.restype = ct.c_double
        L.bdo_zeitschritte.argtypes = [ct.c_void_p, ct.c_int]
        L.bdo_zeitschritte.restype = ct.c_double
        L.bdo_zeitschritt_mrd.argtypes = [ct.c_void_p, ct.c_double]
        L.bdo_zeitschritt_mrd.restype = ct.c_double
        L.bdo_init_positions.argtypes = [ct.c_void_p, ct.c_int]
        L.bdo_set_positions.argtypes = [ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_void_p]
        L.bdo_get_positions.argtypes = [ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_void_p]
        L.bdo_get_forces.argtypes = [ct.c_void_p, ct.c_int, ct.c_int, ct.c_void_p]
        L.bdo_get_grid.argtypes = [ct.c_void_p, ct.c_int, ct.c_void_p]
        L.bdo_get_list.argtypes = [ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, ct.c_void_p, ct.c_int]
        L.bdo_get_list.restype = ct.c_int
        L.bdo_oob_count.argtypes = [ct.c_void_p]
        L.bdo_oob_count.restype = ct.c_long
        L.bdo_set_noise.argtypes = [ct.c_void_p, ct.c_int, ct.c_uint64]
        L.bdo_inject_uniforms.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_size_t]
        L.bdo_set_step.argtypes = [ct.c_void_p, ct.c_uint64]
        L.bdo_get_step.argtypes = [ct.c_void_p]
        L.bdo_get_step.restype = ct.c_uint64
        L.bdo_philox_noise.argtypes = [ct.c_uint64, ct.c_uint64, ct.c_int, ct.c_int, ct.c_int,
                                       ct.c_void_p, ct.c_void_p]
        L.bdo_philox4x32_10.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_void_p]
        L.bdo_nachList_Zellen.argtypes = [ct.c_void_p]
        L.bdo_nachList_Zellen.restype = ct.c_int
        L.bdo_nachList_Breite.argtypes = [ct.c_void_p]
        L.bdo_nachList_Breite.restype = ct.c_double
        L.bdo_uniform.argtypes = [ct.c_void_p]
        L.bdo_uniform.restype = ct.c_double
        L.bdo_schreibe_pos.argtypes = [ct.c_void_p, ct.c_char_p, ct.c_char_p, ct.c_int, ct.c_int]
        L.bdo_schreibe_pos.restype = ct.c_int
        L.bdo_snapgrid_num.argtypes = [ct.c_double, ct.c_double]
        L.bdo_snapgrid_num.restype = ct.c_int
        L.bdo_lokale_dichte.argtypes = [ct.c_int, ct.c_double, ct.c_int, ct.c_void_p, ct.c_int,
                                         ct.c_void_p, ct.c_void_p, ct.c_void_p]
        L.bdo_rhohist.argtypes = [ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_double,
                                  ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ct.c_void_p)


def to_params(p):
    s = BdoParams()
    for name, typ in BdoParams._fields_:
        v = p[name]
        setattr(s, name, int(v) if typ is ct.c_int else float(v))
    return s


class Oracle:
    """FP64 restatement of the reference's RunDynamik for one run."""

    def __init__(self, params, seed=0):
        self.p = dict(params)
        self._params = to_params(self.p)
        self.L = lib()
        self.h = self.L.bdo_create(ct.byref(self._params), seed)
        self.N = (self.p["N1"], self.p["N2"])
        self.Z = self.p["FFT_samples"]
        self.C = self.L.bdo_nachList_Zellen(self.h)
        self.B = self.L.bdo_nachList_Breite(self.h)
        self._keep = None

    def __del__(self):
        if getattr(self, "h", None):
            self.L.bdo_destroy(self.h)
            self.h = None

    def init_positions(self, methode=1):
        r = self.L.bdo_init_positions(self.h, methode)
        if r != 0:
            raise ValueError("init method %d not applicable" % methode)

    def set_positions(self, pos):
        """pos: dict species -> (git int32[N,2], rel float64[N,2])"""
        for s in (0, 1):
            g, r = pos[s]
            g = np.ascontiguousarray(g, dtype=np.int32)
            r = np.ascontiguousarray(r, dtype=np.float64)
            self.L.bdo_set_positions(self.h, s, _ptr(g), _ptr(r))
        self.L.bdo_WCA_init(self.h)

    def get_positions(self):
        out = {}
        for s in (0, 1):
            g = np.zeros((self.N[s], 2), np.int32)
            r = np.zeros((self.N[s], 2), np.float64)
            self.L.bdo_get_positions(self.h, s, _ptr(g), _ptr(r))
            out[s] = (g, r)
        return out

    def forces(self):
        """Reference order: WCA11, WCA22, WCA12, capillary."""
        self.L.bdo_berechne_WCA11(self.h)
        self.L.bdo_berechne_WCA22(self.h)
        self.L.bdo_addiere_WCA12(self.h)
        self.L.bdo_berechne_kapkraefte(self.h)
        return self.get_forces()

    def get_forces(self):
        out = {}
        for kind, name in ((0, "wca"), (1, "kap"), (2, "noise")):
            for s in (0, 1):
                a = np.zeros((self.N[s], 2))
                self.L.bdo_get_forces(self.h, kind, s, _ptr(a))
                out[(name, s)] = a
        return out

    def grid(self, which):
        a = np.zeros(self.Z * self.Z)
        self.L.bdo_get_grid(self.h, which, _ptr(a))
        return a.reshape(self.Z, self.Z)

    def list(self, species, i, j):
        n = self.L.bdo_get_list(self.h, species, i, j, None, 0)
        a = np.zeros(max(n, 1), np.int32)
        self.L.bdo_get_list(self.h, species, i, j, _ptr(a), n)
        return a[:n]

    def set_noise(self, mode, seed=0):
        self.L.bdo_set_noise(self.h, mode, seed)

    def inject(self, u):
        self._keep = np.ascontiguousarray(u, dtype=np.float64)
        self.L.bdo_inject_uniforms(self.h, _ptr(self._keep), self._keep.size)

    def set_step(self, step):
        self.L.bdo_set_step(self.h, step)

    def step(self, n=1):
        return self.L.bdo_zeitschritte(self.h, n)

    def step_mrd(self, mrd):
        """One step with travel bound mrd (zeitschritt_debug's step length)."""
        return self.L.bdo_zeitschritt_mrd(self.h, mrd)

    def oob(self):
        return self.L.bdo_oob_count(self.h)

    def optimaler_zeitschritt(self):
        return self.L.bdo_optimaler_zeitschritt(self.h)

    def schreibe_pos(self, path1, path2, nr, header):
        return self.L.bdo_schreibe_pos(self.h, path1.encode(), path2.encode(), nr, int(header))


# local densities of the offline analysis (main_auswertung.cpp:182-390)
RHOHIST_BINS, RHOHIST_DRHO = 100, 0.01                      # parameter.h:109-110
RHO_THRESH = (0.1, 0.2, 0.5)                                # parameter.h:117-119
DRHO_THRESH = (0.1, 0.2, 0.5, 0.99)                         # parameter.h:121-124
SNAPGRID_CRUDE = 0.5                                        # parameter.h:161


def snapgrid_num(L, crude=SNAPGRID_CRUDE):
    return lib().bdo_snapgrid_num(float(L), float(crude))


def lokale_dichte(L, x1, x2, crude=SNAPGRID_CRUDE):
    """TSC-gridded densities (g1, g2) of absolute positions x1, x2 [N, 2]."""
    n = snapgrid_num(L, crude)
    x1 = np.ascontiguousarray(x1, np.float64).reshape(-1, 2)
    x2 = np.ascontiguousarray(x2, np.float64).reshape(-1, 2)
    g1, g2 = np.zeros(n * n), np.zeros(n * n)
    lib().bdo_lokale_dichte(n, L / n, len(x1), _ptr(x1), len(x2), _ptr(x2), _ptr(g1), _ptr(g2))
    return g1.reshape(n, n), g2.reshape(n, n)


def rhohist(g1, g2, bins=RHOHIST_BINS, dbin=RHOHIST_DRHO, rho_thresh=RHO_THRESH,
            drho_thresh=DRHO_THRESH):
    """(hist int[4, bins] = rho1, rho2, rho, drho counts; over int[7])."""
    g1 = np.ascontiguousarray(g1, np.float64)
    g2 = np.ascontiguousarray(g2, np.float64)
    rt = np.array(rho_thresh, np.float64)
    dt = np.array(drho_thresh, np.float64)
    hist = np.zeros((4, bins), np.int32)
    over = np.zeros(7, np.int32)
    lib().bdo_rhohist(g1.shape[0], _ptr(g1), _ptr(g2), bins, dbin, _ptr(rt), _ptr(dt), _ptr(hist),
                      _ptr(over))
    return hist, over


def philox_noise(seed, step, N1, N2, gauss=False, with_u=False):
    xi = np.zeros((N1 + N2, 2))
    u = np.zeros((N1 + N2, 2)) if with_u else None
    lib().bdo_philox_noise(seed, step, N1, N2, int(gauss), _ptr(xi),
                           _ptr(u) if with_u else None)
    return (xi, u) if with_u else xi


# ---------------------------------------------------------------------------
# compiled reference checker (oracle/_ref/<config>/bdref)

def ref_exe(name):
    return os.path.join(HERE, "_ref", name, "bdref")


def have_ref(name):
    return os.path.exists(ref_exe(name))


def write_pos(path, pos):
    with open(path, "wb") as f:
        f.write(np.array([len(pos[0][0]), len(pos[1][0])], np.int32).tobytes())
        for s in (0, 1):
            f.write(np.ascontiguousarray(pos[s][0], np.int32).tobytes())
            f.write(np.ascontiguousarray(pos[s][1], np.float64).tobytes())


def _read_pos_from(buf, off):
    n1, n2 = np.frombuffer(buf, np.int32, 2, off)
    off += 8
    out = {}
    for s, n in ((0, n1), (1, n2)):
        g = np.frombuffer(buf, np.int32, 2 * n, off).reshape(n, 2).copy()
        off += 8 * n
        r = np.frombuffer(buf, np.float64, 2 * n, off).reshape(n, 2).copy()
        off += 16 * n
        out[s] = (g, r)
    return out, off


def read_pos(path):
    return _read_pos_from(open(path, "rb").read(), 0)[0]


def _run(args, cwd):
    r = subprocess.run(args, cwd=cwd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("reference checker failed: %s\n%s" % (args, r.stderr[-2000:]))
    return r.stdout


def ref_init(name, seed):
    with tempfile.TemporaryDirectory() as d:
        _run([ref_exe(name), "init", str(seed), os.path.join(d, "a.pos")], d)
        return read_pos(os.path.join(d, "a.pos"))


def ref_forces(name, pos, Z):
    with tempfile.TemporaryDirectory() as d:
        write_pos(os.path.join(d, "in.pos"), pos)
        out = _run([ref_exe(name), "forces", os.path.join(d, "in.pos"), os.path.join(d, "o.bin")], d)
        buf = np.fromfile(os.path.join(d, "o.bin"), np.float64)
    n1, n2 = len(pos[0][0]), len(pos[1][0])
    o = 0
    res = {}
    for key, n in ((("wca", 0), n1), (("kap", 0), n1), (("wca", 1), n2), (("kap", 1), n2)):
        res[key] = buf[o:o + 2 * n].reshape(n, 2)
        o += 2 * n
    for name_ in ("rho", "Fx", "Fy", "Fx_im"):
        res[name_] = buf[o:o + Z * Z].reshape(Z, Z)
        o += Z * Z
    res["oob_messages"] = out.count("Index out of Bounds")
    return res


def ref_steps(name, pos, nsteps, every, noise_u=None):
    """Run zeitschritt() nsteps times. noise_u: float64[nsteps, N1+N2, 2] of
    injected uniforms, or None for the seeded reference stream."""
    with tempfile.TemporaryDirectory() as d:
        write_pos(os.path.join(d, "in.pos"), pos)
        nf = "-"
        if noise_u is not None:
            nf = os.path.join(d, "noise.bin")
            np.ascontiguousarray(noise_u, np.float64).tofile(nf)
        out = _run([ref_exe(name), "steps", os.path.join(d, "in.pos"), str(nsteps), nf,
                    str(every), os.path.join(d, "o.bin")], d)
        buf = open(os.path.join(d, "o.bin"), "rb").read()
    recs = []
    off = 0
    while off < len(buf):
        t = np.frombuffer(buf, np.float64, 1, off)[0]
        off += 8
        p, off = _read_pos_from(buf, off)
        recs.append((t, p))
    return recs, out.count("Index out of Bounds")


def ref_lists(name, pos, C):
    with tempfile.TemporaryDirectory() as d:
        write_pos(os.path.join(d, "in.pos"), pos)
        _run([ref_exe(name), "lists", os.path.join(d, "in.pos"), os.path.join(d, "o.bin")], d)
        buf = np.fromfile(os.path.join(d, "o.bin"), np.int32)
    lists = [dict(), dict()]
    o = 0
    for s in (0, 1):
        for i in range(C):
            for j in range(C):
                n = buf[o]
                o += 1
                lists[s][(i, j)] = buf[o:o + n].copy()
                o += n
    return lists


def ref_time(name, seed, nsteps, warmup):
    import json
    with tempfile.TemporaryDirectory() as d:
        out = _run([ref_exe(name), "time", str(seed), str(nsteps), str(warmup)], d)
    for line in out.splitlines():
        if line.startswith("{"):
            return json.loads(line)
    raise RuntimeError("no timing line from reference checker")


def absolute(pos, B):
    """Absolute coordinates x = git*B + rel per species."""
    return {s: pos[s][0] * B + pos[s][1] for s in (0, 1)}


def nonoverlap_positions(params, seed, dmin=0.95, max_tries=200):
    """Seeded uniform-random positions with a minimum pair distance (random
    sequential addition), in the reference layout with cells from floor(x/B).
    Used for trajectory comparisons, where the reference's fixed-dt updates
    of overlapping random starts move particles by several cells per step."""
    rng = np.random.default_rng(seed)
    L = params["L"]
    N = params["N1"] + params["N2"]
    import math
    C = int(math.floor(L / 2 ** (1 / 6)))
    B = L / C
    ncell = max(1, int(L // dmin))
    cw = L / ncell
    grid = {}
    pts = np.zeros((N, 2))
    k = 0
    while k < N:
        for _ in range(max_tries):
            x, y = rng.uniform(0, L, 2)
            cx, cy = int(x / cw) % ncell, int(y / cw) % ncell
            ok = True
            for ddx in (-1, 0, 1):
                for ddy in (-1, 0, 1):
                    for q in grid.get(((cx + ddx) % ncell, (cy + ddy) % ncell), ()):
                        dx = x - pts[q, 0]
                        dy = y - pts[q, 1]
                        dx -= L * round(dx / L)
                        dy -= L * round(dy / L)
                        if dx * dx + dy * dy < dmin * dmin:
                            ok = False
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if ok:
                pts[k] = (x, y)
                grid.setdefault((cx, cy), []).append(k)
                k += 1
                break
        else:
            raise RuntimeError("could not place particle %d" % k)
    g = np.floor(pts / B).astype(np.int32) % C
    r = pts - g * B
    n1 = params["N1"]
    return {0: (g[:n1].copy(), r[:n1].copy()), 1: (g[n1:].copy(), r[n1:].copy())}


# ---------------------------------------------------------------------------
# the reference's offline analysis program (oracle/_ref/<config>_auswertung/)

def auswertung_exe(name):
    return os.path.join(HERE, "_ref", name + "_auswertung", "auswertung")


def _table(path, float_text=False):
    """Numeric rows of a whitespace-separated text file, frames split at
    blank lines; comment lines are skipped. float_text: parse each value to
    single precision with the C library's strtof first."""
    frames, cur = [], []
    conv = float
    if float_text:
        libc = ct.CDLL(None)
        libc.strtof.restype = ct.c_float
        libc.strtof.argtypes = [ct.c_char_p, ct.c_void_p]
        conv = lambda v: float(libc.strtof(v.encode(), None))
    for line in open(path):
        s = line.strip()
        if s.startswith("#"):
            continue
        if not s:
            if cur:
                frames.append(np.array(cur))
                cur = []
            continue
        cur.append([conv(v) for v in s.split()])
    if cur:
        frames.append(np.array(cur))
    return frames


def ref_auswertung(name, frames):
    """Run the reference's main_auswertung on position frames (a list of
    pos dicts as set_positions takes), written as RunObs::schreibe_pos
    writes them. Returns per frame: the absolute positions it read back
    (x1, x2 as float64 of the float text values), its gridded densities
    (g1, g2 [n, n] as printed), histogram counts hist [4, bins] (rho1,
    rho2, rho, drho) and threshold counts over [7], recovered from the
    printed fractions."""
    from configs import CONFIGS
    p = CONFIGS[name]
    exe = auswertung_exe(name)
    out = []
    with tempfile.TemporaryDirectory() as d:
        o = Oracle(p, 0)
        p1, p2 = os.path.join(d, "pos1_1.txt"), os.path.join(d, "pos2_1.txt")
        for nr, pos in enumerate(frames):
            o.set_positions(pos)
            o.schreibe_pos(p1, p2, nr, nr == 0)
        os.makedirs(os.path.join(d, "localDens"))
        _run([exe], d)
        # the reference reads the positions with fscanf("%g") into float
        # (main_auswertung.cpp:103-131): parse them the same way, with strtof
        xs = [_table(p1, float_text=True), _table(p2, float_text=True)]
        rh, dh = _table(os.path.join(d, "rhoHist.txt")), _table(os.path.join(d, "drhoHist.txt"))
        rt, dt = _table(os.path.join(d, "rhoThresh.txt")), _table(os.path.join(d, "drhoThresh.txt"))
        for t in range(len(frames)):
            g = _table(os.path.join(d, "localDens", "rho%d.txt" % t))[0]
            n = int(round(np.sqrt(len(g))))
            cells = n * n
            hist = np.stack([rh[t][:, 2], rh[t][:, 3], rh[t][:, 4], dh[t][:, 2]]) * cells
            over = np.concatenate([rt[0][t, 1:], dt[0][t, 1:]]) * cells
            out.append(dict(x1=xs[0][t][:, 1:], x2=xs[1][t][:, 1:],
                            g1=g[:, 3].reshape(n, n), g2=g[:, 4].reshape(n, n),
                            hist=np.rint(hist).astype(np.int32), over=np.rint(over).astype(np.int32)))
    return out


def ref_obs(name, pos):
    """The reference's in-run observables on `pos` (RunObs::record_
    korrelationsfunktion11/12/22 and record_ftrho_unkorrigiert,
    auswertung.cpp:110-188, 262-375): dict with g11, g12, g22 [korr_bins]
    and, per distinct |q|^2 = i^2 + j^2 in order of first appearance
    (qabs2), the sums re/im of exp(i k.r) over the (i, j) with that |q|^2
    for species 1 and 2 (ftrho1_re, ftrho1_im, ftrho2_re, ftrho2_im)."""
    with tempfile.TemporaryDirectory() as d:
        write_pos(os.path.join(d, "in.pos"), pos)
        _run([ref_exe(name), "obs", os.path.join(d, "in.pos"), os.path.join(d, "o.bin")], d)
        buf = open(os.path.join(d, "o.bin"), "rb").read()
    kb = int(np.frombuffer(buf, np.int32, 1, 0)[0])
    off = 4
    out = {}
    for k in ("g11", "g12", "g22"):
        out[k] = np.frombuffer(buf, np.float64, kb, off).copy()
        off += 8 * kb
    nq = int(np.frombuffer(buf, np.int32, 1, off)[0])
    off += 4
    out["qabs2"] = np.frombuffer(buf, np.int32, nq, off).copy()
    off += 4 * nq
    for k in ("ftrho1_re", "ftrho1_im", "ftrho2_re", "ftrho2_im"):
        out[k] = np.frombuffer(buf, np.float64, nq, off).copy()
        off += 8 * nq
    return out
