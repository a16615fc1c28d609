"""Host-side logic of libbd_b200.so on CPU: parameters and the parameter.h
reader, the reference's initialisers (bit-exact against the reference's own
output), the pos-file format, and the exported C ABI."""
import os
import re

import numpy as np
import pytest

import configs as C
from conftest import ROOT, golden, gpos


def test_every_declared_symbol_is_exported(bdsim_mod):
    hdr = open(os.path.join(ROOT, "include", "bd_api.h")).read()
    declared = set(re.findall(r"\b(bd_[A-Za-z0-9_]+)\s*\(", hdr))
    L = bdsim_mod.lib()
    missing = [n for n in sorted(declared) if not hasattr(L, n)]
    assert not missing, missing
    assert declared == set(bdsim_mod.EXPORTS)


def test_defaults_are_parameter_h(bdsim_mod):
    p = bdsim_mod.default_params()
    for k, v in C.param_defaults().items():
        if hasattr(p, k):
            assert float(getattr(p, k)) == pytest.approx(float(v)), k
    assert p.noise_kind == bdsim_mod.NOISE_DISK and p.ngp_ref_compat == 1


def test_reference_parameter_h_parses(bdsim_mod):
    """The reference's shipped parameter.h, found where oracle/build_ref.py
    looks for the reference (BD_REFERENCE_DIR)."""
    import build_ref
    path = os.path.join(build_ref.REF, "parameter.h")
    if not os.path.exists(path):
        pytest.skip("reference sources not present")
    p = bdsim_mod.params_from_header(path)
    for k, v in C.param_defaults().items():
        if hasattr(p, k):
            assert float(getattr(p, k)) == pytest.approx(float(v)), k


def test_header_expressions(bdsim_mod, tmp_path):
    f = tmp_path / "parameter.h"
    f.write_text("""
// comment
#pragma once
const int N1 = 123; /* block
comment */
const int N2 = 2*N1 + 1;
const double L = 40.0;
const double sigma11_22 = 1.5;
const double sigma11_12 = 0.5*(1.0 + sigma11_22);
const double lambda_kapillar = 3.0;
const double startpos_kreisradius = 4.5 * lambda_kapillar;
const double f2_f1 = - 1.0;
const bool idgas_only = true;
const int FFT_samples = 2 * (int) (L/2.5 + 0.5);
const string startpos_dateiname="startpos.txt";
const double zweihoch1_6 = pow(2.0, 1.0/6.0);
const int nachList_Zellen = (int) floor(L/zweihoch1_6);
""")
    p = bdsim_mod.params_from_header(str(f))
    assert p.N1 == 123 and p.N2 == 247
    assert p.sigma11_12 == pytest.approx(1.25)
    assert p.startpos_kreisradius == pytest.approx(13.5)
    assert p.f2_f1 == -1.0 and p.idgas_only == 1
    assert p.FFT_samples == 32


@pytest.mark.parametrize("name", ["tiny_cic", "tiny_tsc", "c1_cic", "ref_default", "tiny_radial"])
def test_derived_constants(bdsim_mod, name):
    p = bdsim_mod.params_from(C.CONFIGS[name])
    d = bdsim_mod.derived(p)
    ref = C.derived(C.CONFIGS[name])
    assert d.nachList_Zellen == ref["nachList_Zellen"]
    assert d.nachList_Breite == ref["nachList_Breite"]
    assert d.densGrid_Breite == ref["densGrid_Breite"]
    assert d.fixed_dt == (C.CONFIGS[name]["max_reisedistanz"] >= 1e20)


@pytest.mark.parametrize("name", ["tiny_ngp", "tiny_cic", "tiny_tsc", "c1_cic", "ref_default", "tiny_radial"])
def test_library_initialisers_match_reference(bdsim_mod, name):
    """The library's host initialisers reproduce the reference's starting
    positions bit for bit (init_zufallspos incl. Q4; init_kernundring)."""
    p = C.CONFIGS[name]
    pos = bdsim_mod.init_positions_host(bdsim_mod.params_from(p), 7, p["startpos_methode"])
    ref = gpos(golden(name), "init")
    for s in (0, 1):
        assert np.array_equal(pos[s][0], ref[s][0])
        assert np.array_equal(pos[s][1], ref[s][1])


@pytest.mark.parametrize("methode", [1, 4, 5])
def test_other_initialisers_match_oracle(bdsim_mod, oracle_mod, methode):
    p = dict(C.CONFIGS["tiny_cic"], startpos_kreisradius=12.0)  # disk inside the box
    pos = bdsim_mod.init_positions_host(bdsim_mod.params_from(p), 99, methode)
    o = oracle_mod.Oracle(p, 99)
    o.init_positions(methode)
    ref = o.get_positions()
    for s in (0, 1):
        assert np.array_equal(pos[s][0], ref[s][0])
        assert np.array_equal(pos[s][1], ref[s][1])


def test_grid_and_forcetest_initialisers(bdsim_mod, oracle_mod):
    p = dict(C.CONFIGS["tiny_cic"], N1=50, N2=0)
    a = bdsim_mod.init_positions_host(bdsim_mod.params_from(p), 1, 3)
    o = oracle_mod.Oracle(p, 1)
    o.init_positions(3)
    b = o.get_positions()
    assert np.array_equal(a[0][0], b[0][0]) and np.array_equal(a[0][1], b[0][1])
    p = dict(C.CONFIGS["tiny_cic"], N1=2, N2=0)
    a = bdsim_mod.init_positions_host(bdsim_mod.params_from(p), 1, 7)
    o = oracle_mod.Oracle(p, 1)
    o.init_positions(7)
    b = o.get_positions()
    assert np.array_equal(a[0][0], b[0][0]) and np.array_equal(a[0][1], b[0][1])


def test_pos_file_format_byte_exact(bdsim_mod, oracle_mod, tmp_path):
    """schreibe_pos text (auswertung.cpp:631-648) on identical doubles."""
    p = C.CONFIGS["tiny_cic"]
    g = golden("tiny_cic")
    pos = gpos(g, "init")
    o = oracle_mod.Oracle(p, 1)
    o.set_positions(pos)
    o.schreibe_pos(str(tmp_path / "o1.txt"), str(tmp_path / "o2.txt"), 0, True)
    o.schreibe_pos(str(tmp_path / "o1.txt"), str(tmp_path / "o2.txt"), 3, False)
    B = C.derived(p)["nachList_Breite"]
    for s, name in ((0, "l1.txt"), (1, "l2.txt")):
        path = str(tmp_path / name)
        bdsim_mod.write_pos_frame(path, False, 0.0, pos[s][0], pos[s][1], B)
        bdsim_mod.write_pos_frame(path, True, 3 * p["obs_dt"], pos[s][0], pos[s][1], B)
    assert (tmp_path / "l1.txt").read_bytes() == (tmp_path / "o1.txt").read_bytes()
    assert (tmp_path / "l2.txt").read_bytes() == (tmp_path / "o2.txt").read_bytes()


def test_unsupported_parameters_rejected(bdsim_mod):
    L = bdsim_mod.lib()
    import ctypes as ct
    n = ct.c_size_t()
    bad = [dict(C.CONFIGS["tiny_cic"], L=3.0),           # fewer than 3 cells per side
           dict(C.CONFIGS["tiny_cic"], FFT_samples=40),  # 40 = 2^3 * 5
           dict(C.CONFIGS["tiny_cic"], N1=0),
           dict(C.CONFIGS["tiny_cic"], densGrid_Schema=3)]
    for q in bad:
        assert L.bd_run_footprint(ct.byref(bdsim_mod.params_from(q)), ct.byref(n)) < 0


def test_create_without_device_fails_loudly(bdsim_mod):
    if bdsim_mod.device_count() > 0:
        pytest.skip("a CUDA device is present")
    with pytest.raises(bdsim_mod.BdError) as e:
        bdsim_mod.Run(C.CONFIGS["tiny_cic"])
    assert e.value.status == -2


def test_autotune_argument_checks(bdsim_mod):
    """bd_batch_autotune rejects a missing batch, a missing result and
    reps <= 0 before touching a device (BD_ERR_ARG)."""
    import ctypes as ct
    L = bdsim_mod.lib()
    res = bdsim_mod.TuneResult()
    assert L.bd_batch_autotune(None, 3, ct.byref(res)) == -1
    assert L.bd_batch_autotune(ct.c_void_p(1), 3, None) == -1
    assert L.bd_batch_autotune(ct.c_void_p(1), 0, ct.byref(res)) == -1


def test_step_form_argument_checks(bdsim_mod):
    """bd_batch_set_step_form rejects a missing batch, an unknown form and
    CTAs per SM outside its form's range before touching a device."""
    import ctypes as ct
    L = bdsim_mod.lib()
    assert L.bd_batch_set_step_form(None, 0, 0) == -1
    for form, ctas in ((2, 0), (-1, 0), (0, 3), (1, 1), (1, 5), (1, -1)):
        assert L.bd_batch_set_step_form(ct.c_void_p(1), form, ctas) == -1, (form, ctas)


def test_lokdens_params_default_and_header(bdsim_mod, tmp_path):
    """The analysis program's constants (parameter.h:109-124,161) and
    snapgrid_num (parameter.h:174), through the C ABI."""
    lp = bdsim_mod.lokdens_params()
    assert (lp.snapgrid_crude, lp.rhohist_bins, lp.rhohist_drho) == (0.5, 100, 0.01)
    assert list(lp.rho_thresh) == [0.1, 0.2, 0.5] and list(lp.drho_thresh) == [0.1, 0.2, 0.5, 0.99]
    f = tmp_path / "parameter.h"
    f.write_text("""
const int rhohist_bins = 40;
const double rhohist_drho = 0.05;
const double rho_thresh1 = 0.3, rho_thresh2 = 0.4, rho_thresh3 = 2*rho_thresh2;
const double drho_thresh4= 0.9;
const double snapgrid_crude = 1.25;
""")
    lp = bdsim_mod.lokdens_params_from_header(str(f))
    assert (lp.snapgrid_crude, lp.rhohist_bins, lp.rhohist_drho) == (1.25, 40, 0.05)
    assert list(lp.rho_thresh) == [0.3, 0.4, 0.8] and list(lp.drho_thresh) == [0.1, 0.2, 0.5, 0.9]
    ct = __import__("ctypes")
    for L, crude in ((40.0, 0.5), (36.0, 0.5), (2896.0, 0.5), (100.0, 0.7), (3.0, 2.0)):
        n = ct.c_int()
        p = bdsim_mod.params_from(dict(C.CONFIGS["tiny_cic"], L=L))
        st = bdsim_mod.lib().bd_snapgrid_num(ct.byref(p), ct.byref(bdsim_mod.lokdens_params(snapgrid_crude=crude)),
                                             ct.byref(n))
        assert st == 0 and n.value == 2 * int(L / (2 * crude) + 0.5)
    n = ct.c_int()
    assert bdsim_mod.lib().bd_snapgrid_num(ct.byref(p), ct.byref(bdsim_mod.lokdens_params(snapgrid_crude=0.0)),
                                           ct.byref(n)) == -1


def test_ctypes_structs_match_the_c_header(bdsim_mod, tmp_path):
    """Every struct the ctypes binding mirrors has the size and field offsets
    the C compiler gives it from include/bd_api.h."""
    import ctypes as ct
    import subprocess
    pairs = {"bd_params": bdsim_mod.Params, "bd_derived": bdsim_mod.Derived,
             "bd_timestep_info": bdsim_mod.TimestepInfo, "bd_lokdens_params": bdsim_mod.LokDensParams,
             "bd_serve_opts": bdsim_mod.ServeOpts, "bd_req_status": bdsim_mod.ReqStatus,
             "bd_serve_stats": bdsim_mod.ServeStats, "bd_tune_result": bdsim_mod.TuneResult}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "bd_api.h"', "int main(void) {"]
    for cname, py in pairs.items():
        lines.append('printf("%s size %%zu\\n", sizeof(%s));' % (cname, cname))
        for fname, _ in py._fields_:
            lines.append('printf("%s %s %%zu\\n", offsetof(%s, %s));' % (cname, fname, cname, fname))
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {}
    for line in out:
        if line:
            a, b, c = line.split()
            got[(a, b)] = int(c)
    for cname, py in pairs.items():
        assert got[(cname, "size")] == ct.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)
