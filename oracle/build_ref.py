"""Build recipe for the compiled reference checker (test infrastructure).

Compiles the reference's own step translation units where they lie under
/root/reference (reference Makefile:7 minus main.cpp and zufall.cpp), with the
reference's flags `-O3 -std=c++0x -fopenmp` (Makefile:2,5), once per named
configuration, into oracle/_ref/<config>/bdref. Nothing from the reference is
copied; only build outputs are written, and only under oracle/_ref/.

Three link-time substitutions make it runnable here:
  * parameter.h: the reference hard-codes every parameter as a compile-time
    const (parameter.h:14-209). A generated parameter.h with the same names is
    written to oracle/_ref/<config>/ and found first through `-I<dir> -I-`
    (`-I-` stops the quoted-include search from starting in the including
    file's own directory).
  * FFTW3 is not installed; oracle/fftw_shim provides the FFTW3 calls used.
  * zufall.cpp is replaced by oracle/ref_seam.cpp (seedable, injectable RNG);
    `-include ctime` is not needed because zufall.cpp is not compiled (it uses
    time() without <ctime>, which g++ 13 rejects).
oracle/ref_harness.cpp replaces main.cpp.

Usage: python oracle/build_ref.py [config ...]   (default: every REF_BUILDS entry)
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from configs import CONFIGS, REF_BUILDS  # noqa: E402

REF = os.environ.get("BD_REFERENCE_DIR", "/root/reference")
OUT = os.path.join(HERE, "_ref")
REF_TUS = ["dynamik_methoden.cpp", "gridRoutinen.cpp", "allgemeine_methoden.cpp",
           "auswertung.cpp"]
FLAGS = ["-O3", "-std=c++0x", "-fopenmp", "-w"]


def _b(v):
    return "true" if v else "false"


def parameter_h(p):
    """parameter.h with the reference's names; derived constants follow the
    reference's own formulas (parameter.h:171-209)."""
    r = repr
    lines = [
        "// generated for the compiled reference checker; names as reference parameter.h",
        "#pragma once",
        "#define _USE_MATH_DEFINES",
        "#include <math.h>",
        "#include <string>",
        "using std::string;",
        f"const int N1 = {p['N1']};",
        f"const int N2 = {p['N2']};",
        f"const double L = {r(float(p['L']))};",
        f"const int densGrid_Schema = {p['densGrid_Schema']};",
        f"const int FFT_samples = {p['FFT_samples']};",
        f"const double lambda_kapillar = {r(float(p['lambda_kapillar']))};",
        f"const double kapillar_vorfaktor = {r(float(p['kapillar_vorfaktor']))};",
        f"const double T = {r(float(p['T']))};",
        f"const double dt_max = {r(float(p['dt_max']))};",
        f"const double max_reisedistanz = {r(float(p['max_reisedistanz']))};",
        f"const double sigma11_22 = {r(float(p['sigma11_22']))};",
        f"const double sigma11_12 = {r(float(p['sigma11_12']))};",
        f"const double Gamma2_1 = {r(float(p['Gamma2_1']))};",
        f"const double eps22_11 = {r(float(p['eps22_11']))};",
        f"const double eps12_11 = {r(float(p['eps12_11']))};",
        f"const double f2_f1 = {r(float(p['f2_f1']))};",
        f"const bool idgas_only = {_b(p['idgas_only'])};",
        f"const bool noWCA = {_b(p['noWCA'])};",
        f"const bool noRNG = {_b(p['noRNG'])};",
        f"const bool quickInit = {_b(p['quickInit'])};",
        f"const bool restrictRadial = {_b(p['restrictRadial'])};",
        "const bool debugmode = false;",
        "const bool krafttestmode = false;",
        f"const double maxPairWCA = {r(float(p['maxPairWCA']))};",
        f"const int max_write_interval = {p['max_write_interval']};",
        "const int runs = 1;",
        "const int jobs = 1;",
        "const int maxThreads = 1;",
        f"const double obs_dt = {r(float(p['obs_dt']))};",
        f"const int obs_anzahl = {p['obs_anzahl']};",
        "const double korr_dr = 0.2;",
        "const double korr_rmax = L*0.5;",
        "const int rhohist_bins = 100;",
        "const double rhohist_drho = 0.01;",
        "const double rho_thresh1 = 0.1, rho_thresh2 = 0.2, rho_thresh3 = 0.5;",
        "const double drho_thresh1 = 0.1, drho_thresh2 = 0.2, drho_thresh3 = 0.5, drho_thresh4 = 0.99;",
        "const double rhoring_dr = 0.5;",
        "const int rhoring_bins = 500;",
        "const int ftrho_qbins = 30;",
        f"const int startpos_methode = {p['startpos_methode']};",
        'const string startpos_dateiname = "startpos.txt";',
        f"const double startpos_kreisradius = {r(float(p['startpos_kreisradius']))};",
        'const string pos_output_dateiname = "pos.txt";',
        "const bool auswerten_korrfunk = false;",
        "const bool auswerten_korrfunk_mixed = false;",
        "const bool auswerten_rhovonk = false;",
        "const bool auswerten_rhoviaFFTW = false;",
        "const bool auswerten_rhoFT_normjerun = false;",
        "const bool auswerten_animation = false;",
        "const bool auswerten_abstand = false;",
        "const double snapgrid_crude = 0.5;",
        "const double gaussdens_width_x = 0.1*L;",
        "const double gaussdens_width_y = 0.02*L;",
        # derived, as parameter.h:171-209
        "const double zweihoch1_6 = pow(2.0, 1.0/6.0);",
        "const int snapgrid_num = 2 * (int) (L/(2*snapgrid_crude) + 0.5);",
        "const double snapgrid_width = L / snapgrid_num;",
        "const int nachList_Zellen = (int) floor(L/zweihoch1_6);",
        "const double nachList_Breite = L/((double)nachList_Zellen);",
        "const double densGrid_Breite = L/FFT_samples;",
        "const int densGrid_Zellen = FFT_samples;",
        "const double dq = 2.0*M_PI/L;",
        "const double dq_rhoFFTW = 2.0*dq;",
        "const double dq_dqFT = dq / dq_rhoFFTW;",
        "const int rhoFFTW_bins = 0.5*FFT_samples*dq/dq_rhoFFTW;",
        "const double Omega = M_PI/densGrid_Breite;",
        "const int korr_bins = (int) (korr_rmax/korr_dr)+1;",
        "const double ftrho_dq = 4.0*M_PI/L;",
    ]
    return "\n".join(lines) + "\n"


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: " + " ".join(cmd) + "\n" + r.stderr[-4000:])


def build_one(name, force=False):
    d = os.path.join(OUT, name)
    os.makedirs(d, exist_ok=True)
    exe = os.path.join(d, "bdref")
    ph = os.path.join(d, "parameter.h")
    text = parameter_h(CONFIGS[name])
    own = [os.path.join(HERE, f) for f in ("ref_seam.cpp", "ref_harness.cpp", "build_ref.py",
                                           "bd_oracle.c", "bd_oracle.h",
                                           os.path.join("fftw_shim", "fftw_shim.c"),
                                           os.path.join("fftw_shim", "fftw3.h"))]
    if (not force and os.path.exists(exe) and os.path.exists(ph) and open(ph).read() == text
            and all(os.path.getmtime(s) <= os.path.getmtime(exe) for s in own)):
        return exe
    with open(ph, "w") as f:
        f.write(text)
    shim_o = os.path.join(d, "fftw_shim.o")
    _run(["gcc", "-O3", "-c", os.path.join(HERE, "fftw_shim", "fftw_shim.c"),
          "-I", os.path.join(HERE, "fftw_shim"), "-o", shim_o])
    # the oracle's Philox noise (bdo_philox_noise) for the harness's
    # stepsphilox command: the same uniforms the CUDA library's disk noise uses
    oracle_o = os.path.join(d, "bd_oracle.o")
    _run(["gcc", "-O2", "-std=c99", "-D_GNU_SOURCE", "-ffp-contract=off", "-c",
          os.path.join(HERE, "bd_oracle.c"), "-I", HERE, "-I", os.path.join(HERE, "fftw_shim"),
          "-o", oracle_o])
    srcs = [os.path.join(REF, t) for t in REF_TUS]
    srcs += [os.path.join(HERE, "ref_seam.cpp"), os.path.join(HERE, "ref_harness.cpp")]
    _run(["g++"] + FLAGS + ["-I" + d, "-I-", "-I" + os.path.join(HERE, "fftw_shim"),
                            "-I" + REF] + srcs + [shim_o, oracle_o, "-lm", "-o", exe])
    return exe


def build_auswertung(name, frames, force=False):
    """The reference's offline analysis program (main_auswertung.cpp, built
    as Makefile:23-24 does, `g++ main_auswertung.cpp -O3`, in the C++11 mode of
    Makefile:2 so that `-I-` does not hide libstdc++'s own headers) for configuration
    `name` with obs_anzahl = frames, into oracle/_ref/<name>_auswertung/.
    It reads pos1_1.txt / pos2_1.txt from its working directory and writes
    korrfunk_run1.txt, localDens/rho<t>.txt, rhoHist.txt, drhoHist.txt,
    rhoThresh.txt and drhoThresh.txt there."""
    d = os.path.join(OUT, name + "_auswertung")
    os.makedirs(d, exist_ok=True)
    exe = os.path.join(d, "auswertung")
    ph = os.path.join(d, "parameter.h")
    text = parameter_h(dict(CONFIGS[name], obs_anzahl=frames))
    if (not force and os.path.exists(exe) and os.path.exists(ph) and open(ph).read() == text
            and os.path.getmtime(os.path.abspath(__file__)) <= os.path.getmtime(exe)):
        return exe
    with open(ph, "w") as f:
        f.write(text)
    _run(["g++", "-O3", "-std=c++0x", "-w", "-I" + d, "-I-", "-I" + REF,
          os.path.join(REF, "main_auswertung.cpp"), "-lm", "-o", exe])
    return exe


def build(names=None, jobs=4):
    if not os.path.isdir(REF):
        return []
    names = names or REF_BUILDS
    with ThreadPoolExecutor(jobs) as ex:
        return list(ex.map(build_one, names))


if __name__ == "__main__":
    for e in build(sys.argv[1:] or None):
        print(e)
