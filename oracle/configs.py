"""Named run configurations shared by the oracle build, the tests and bench.py.

Every configuration is a dict of the reference's parameter.h names
(parameter.h:14-165). `param_defaults()` holds the reference's shipped values
(parameter.h:14-139); each named config overrides a few of them.

Mapping of the workload descriptions to reference parameters:
  * WCA sigma = epsilon = 1 for all pairs -> sigma11_22 = sigma11_12 = 1,
    eps22_11 = eps12_11 = 1.
  * capillary pair law -Gamma q_i q_j K0(r/lambda): the mesh Green's function
    1/(q^2 + lambda^-2) is the transform of K0(r/lambda)/(2 pi), so
    kapillar_vorfaktor = 2 pi Gamma and f2_f1 = q2/q1.
  * fixed time step dt: the reference always picks an adaptive step
    (dynamik_methoden.cpp:112) capped at dt_max, so dt_max = dt and a travel
    bound max_reisedistanz = 1e30 that never binds.
  * D = 1: the reference step is dr = dt F + sqrt(2 T dt) xi, so T = D = 1.
"""
import math

# parameter.h:14-139 (values as shipped)
def param_defaults():
    return dict(
        N1=2000, N2=2000, L=300.0, densGrid_Schema=2, FFT_samples=384,
        lambda_kapillar=25.0, kapillar_vorfaktor=1.111111111, T=24.3055555,
        dt_max=0.005, max_reisedistanz=0.24, sigma11_22=1.0, sigma11_12=1.0,
        Gamma2_1=1.0, eps22_11=1.0, eps12_11=1.0, f2_f1=-1.0,
        idgas_only=False, noWCA=False, noRNG=False, quickInit=True,
        restrictRadial=False, debugmode=False, krafttestmode=False,
        maxPairWCA=1.0e5, max_write_interval=900, runs=1, jobs=1, maxThreads=1,
        obs_dt=0.2, obs_anzahl=12, startpos_methode=1,
        startpos_kreisradius=4.5 * 25.0,
    )


TWO_PI = 2.0 * math.pi


def _cfg(**kw):
    p = param_defaults()
    p.update(kw)
    if "startpos_kreisradius" not in kw:
        p["startpos_kreisradius"] = 4.5 * p["lambda_kapillar"]
    return p


CONFIGS = {
    # reference parameter.h as shipped: adaptive dt, TSC on a 384^2 mesh
    # (radix-3 factor), opposite charges f2_f1 = -1
    "ref_default": _cfg(),
    # small uneven cases exercising every routine and flag at oracle speed
    "tiny_ngp": _cfg(N1=300, N2=200, L=40.0, densGrid_Schema=0, FFT_samples=32,
                     lambda_kapillar=5.0, kapillar_vorfaktor=3.0, T=1.5,
                     dt_max=2e-4, max_reisedistanz=1e30, sigma11_22=1.3,
                     sigma11_12=0.5 * (1 + 1.3), eps22_11=0.7, eps12_11=1.2,
                     f2_f1=0.6),
    "tiny_cic": _cfg(N1=300, N2=200, L=40.0, densGrid_Schema=1, FFT_samples=48,
                     lambda_kapillar=5.0, kapillar_vorfaktor=3.0, T=1.5,
                     dt_max=2e-4, max_reisedistanz=1e30, sigma11_22=0.8,
                     sigma11_12=0.9, eps22_11=1.4, eps12_11=0.9, f2_f1=-0.5),
    "tiny_tsc": _cfg(N1=256, N2=256, L=36.0, densGrid_Schema=2, FFT_samples=64,
                     lambda_kapillar=4.0, kapillar_vorfaktor=TWO_PI, T=0.7,
                     dt_max=0.004, max_reisedistanz=0.1, f2_f1=1.0),
    # restrictRadial with the core-and-ring start it is meant for
    # (init_kernundring, ring radius 4.5 lambda)
    "tiny_radial": _cfg(N1=1, N2=60, L=60.0, densGrid_Schema=2, FFT_samples=32,
                        lambda_kapillar=3.0, kapillar_vorfaktor=TWO_PI, T=1.0,
                        dt_max=1e-4, max_reisedistanz=1e30, restrictRadial=True,
                        startpos_methode=6),
    "tiny_flags": _cfg(N1=200, N2=150, L=30.0, densGrid_Schema=1, FFT_samples=32,
                       lambda_kapillar=4.0, kapillar_vorfaktor=TWO_PI, T=1.0,
                       dt_max=1e-4, max_reisedistanz=1e30, noWCA=True),
    "tiny_idgas": _cfg(N1=200, N2=150, L=30.0, densGrid_Schema=2, FFT_samples=32,
                       lambda_kapillar=4.0, kapillar_vorfaktor=TWO_PI, T=1.0,
                       dt_max=1e-4, max_reisedistanz=1e30, idgas_only=True),
    # Plain method, small: L=100, N1=N2=1000, CIC 128^2, lambda=10, Gamma=1,
    # q1=q2=1, D=1, dt=1e-4, 1000 steps
    "c1_cic": _cfg(N1=1000, N2=1000, L=100.0, densGrid_Schema=1, FFT_samples=128,
                   lambda_kapillar=10.0, kapillar_vorfaktor=TWO_PI, T=1.0,
                   dt_max=1e-4, max_reisedistanz=1e30, f2_f1=1.0),
    "c1_ngp": _cfg(N1=1000, N2=1000, L=100.0, densGrid_Schema=0, FFT_samples=128,
                   lambda_kapillar=10.0, kapillar_vorfaktor=TWO_PI, T=1.0,
                   dt_max=1e-4, max_reisedistanz=1e30, f2_f1=1.0),
    "c1_tsc": _cfg(N1=1000, N2=1000, L=100.0, densGrid_Schema=2, FFT_samples=128,
                   lambda_kapillar=10.0, kapillar_vorfaktor=TWO_PI, T=1.0,
                   dt_max=1e-4, max_reisedistanz=1e30, f2_f1=1.0),
    # Single run, medium: L=512, N1=N2=32768, TSC 512^2, lambda=64, q2=0.5,
    # dt=5e-5, 10000 steps
    "c2": _cfg(N1=32768, N2=32768, L=512.0, densGrid_Schema=2, FFT_samples=512,
               lambda_kapillar=64.0, kapillar_vorfaktor=TWO_PI, T=1.0,
               dt_max=5e-5, max_reisedistanz=1e30, f2_f1=0.5),
    # Single run, large: L=2896, N1=N2=2^20, TSC 2048^2, lambda=256, dt=5e-5,
    # 2000 steps
    "c3": _cfg(N1=1048576, N2=1048576, L=2896.0, densGrid_Schema=2,
               FFT_samples=2048, lambda_kapillar=256.0,
               kapillar_vorfaktor=TWO_PI, T=1.0, dt_max=5e-5,
               max_reisedistanz=1e30, f2_f1=1.0),
}

# configs the compiled reference checker is built for
REF_BUILDS = ["ref_default", "tiny_ngp", "tiny_cic", "tiny_tsc", "tiny_radial",
              "tiny_flags", "tiny_idgas", "c1_cic", "c1_ngp", "c1_tsc", "c2", "c3"]

# workload step counts as stated for each single-run config
STEPS = {"c1_cic": 1000, "c2": 10000, "c3": 2000}


def derived(p):
    """Derived constants, computed as parameter.h:171-209 computes them."""
    zweihoch1_6 = 2.0 ** (1.0 / 6.0)
    C = int(math.floor(p["L"] / zweihoch1_6))
    return dict(
        zweihoch1_6=zweihoch1_6,
        nachList_Zellen=C,
        nachList_Breite=p["L"] / float(C),
        densGrid_Breite=p["L"] / p["FFT_samples"],
        densGrid_Zellen=p["FFT_samples"],
        dq=2.0 * math.pi / p["L"],
    )


def batch_ensemble(n_runs=256, seed=2024):
    """Batched ensemble: per-species N log-uniform in [512, 65536], L for an
    area fraction of 0.2 (phi = N_tot * pi/4 / L^2 with sigma = 1), mesh the
    power of two nearest L/2 clamped to [64, 512], NGP/CIC/TSC round-robin,
    lambda = L/8, Gamma = 1, q1 = q2 = 1, D = 1, dt = 5e-5, seeds per run."""
    import numpy as np
    rng = np.random.default_rng(seed)
    runs = []
    for r in range(n_runs):
        n = int(round(math.exp(rng.uniform(math.log(512), math.log(65536)))))
        L = math.sqrt(2 * n * math.pi / (4 * 0.2))
        z = 2 ** int(round(math.log2(L / 2)))
        z = min(max(z, 64), 512)
        runs.append(_cfg(N1=n, N2=n, L=L, densGrid_Schema=r % 3, FFT_samples=z,
                         lambda_kapillar=L / 8, kapillar_vorfaktor=TWO_PI, T=1.0,
                         dt_max=5e-5, max_reisedistanz=1e30, f2_f1=1.0))
    return runs
