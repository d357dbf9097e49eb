"""CPU-only checks of the C ABI library and the host layer (no GPU calls)."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    from amrvac_b200 import build, _lib
    build.build()
    return _lib.load()


def test_library_exports_every_declared_symbol(lib):
    """Every function declared in include/amrvac_gpu.h is exported by the .so."""
    with open(os.path.join(ROOT, "include", "amrvac_gpu.h")) as f:
        text = f.read()
    names = set(re.findall(r"\b(amrvac_(?:gpu|ens|amr)_\w+)\s*\(", text))
    assert len(names) >= 40
    for n in sorted(names):
        assert hasattr(lib, n), n
    from amrvac_b200 import _lib
    assert {s[0] for s in _lib.SIGNATURES} == names


def test_default_cfg_matches_reference_defaults(lib):
    from amrvac_b200 import _lib
    c = _lib.AmrvacCfg()
    lib.amrvac_gpu_default_cfg(ctypes.byref(c))
    assert c.courantpar == 0.8 and c.cada3_radius == 0.1 and c.tvdlfeps == 1.0
    assert c.nghostcells == 2 and list(c.block_nx) == [16, 16, 16]
    assert c.typeboundspeed == 1 and c.mhd_glm_alpha == 0.5 and c.divbdiff == 0.8
    assert c.dtmin == 1e-10 and c.limiter == 1


@pytest.mark.parametrize("ng,nx", [(2, 16), (3, 16), (2, 8), (4, 16)])
def test_srl_maps_match_oracle(lib, oracle_lib, ng, nx):
    from amrvac_b200 import srl_maps
    ours = srl_maps(ng, nx)
    ref = oracle_lib.srl_maps(ng, nx)
    for a, b in zip(ours, ref):
        assert np.array_equal(a, b)


def test_nw(lib):
    from amrvac_b200 import make_cfg
    assert lib.amrvac_gpu_nw(ctypes.byref(make_cfg(physics="hd", ndim=2))) == 4
    assert lib.amrvac_gpu_nw(ctypes.byref(make_cfg(physics="mhd", ndim=3, typedivbfix="glm"))) == 9
    assert lib.amrvac_gpu_nw(ctypes.byref(make_cfg(physics="mhd", ndim=2, ndir=3, typedivbfix="linde"))) == 8


def test_unsupported_configurations_are_refused_without_gpu(lib):
    """Config errors come back as negative codes before any CUDA call."""
    from amrvac_b200 import make_cfg, _lib
    h = ctypes.c_void_p()
    bad = [make_cfg(physics="mhd", ndim=3, typedivbfix="glm", flux_scheme="tvdmu", dimsplit=True),
           make_cfg(physics="hd", ndim=2, flux_scheme="hlld")]
    c = make_cfg(physics="hd", ndim=2)
    c.block_nx[0] = 8  # block_nx must be the same in every direction
    bad.append(c)
    # block edges the library has no kernels for, and what only block_nx 16 runs
    bad += [make_cfg(physics="hd", ndim=2, block_nx=14), make_cfg(physics="hd", ndim=3, block_nx=6),
            make_cfg(physics="hd", ndim=2, block_nx=8, precision="mixed", flux_scheme="tvdlf"),
            make_cfg(physics="hd", ndim=2, block_nx=12, limiter="mp5"),
            make_cfg(physics="mhd", ndim=3, block_nx=10, flux_scheme="tvdmu", dimsplit=True, typedivbfix="glm")]
    # small_values_method: no method 3; 'average' outside its whole-block path
    c = make_cfg(physics="hd", ndim=2, fix_small_values=True)
    c.small_values_method = 3
    bad.append(c)
    avg = dict(fix_small_values=True, small_values_method="average")
    bad += [make_cfg(physics="mhd", ndim=2, typedivbfix="linde", flux_scheme="hll", **avg),
            make_cfg(physics="hd", ndim=2, flux_scheme="tvdlf", time_stepper="twostep", **avg),
            make_cfg(physics="hd", ndim=2, flux_scheme="hll", dimsplit=True, **avg),
            make_cfg(physics="hd", ndim=2, flux_scheme="hll", limiter="venk", **avg)]
    for cfg in bad:
        r = lib.amrvac_gpu_create(ctypes.byref(cfg), ctypes.byref(h))
        assert r == _lib.E_UNSUPPORTED, lib.amrvac_gpu_last_error()
    with pytest.raises(ValueError):
        make_cfg(physics="hd", ndim=2, fix_small_values=True, small_values_method="ignore")


def test_block_nx_from_par_file(tmp_path):
    """block_nx1..3 of &meshlist reach the configuration (the reference's own
    3-D blast test runs 8^3 blocks); unequal edges are refused."""
    from amrvac_b200.config import config_from_par

    def config_from_par_text(text):
        f = tmp_path / "t.par"
        f.write_text(text)
        return config_from_par([str(f)])
    base = """
 &methodlist
        time_stepper = 'threestep'
        flux_scheme = 20*'hll'
        limiter = 20*'koren'
 /
 &meshlist
        domain_nx1=16
        domain_nx2=16
        domain_nx3=16
        block_nx1=8
        block_nx2=8
        block_nx3=%d
 /
 &mhd_list
 /
"""
    rc = config_from_par_text(base % 8)
    assert list(rc.cfg.block_nx) == [8, 8, 8]
    with pytest.raises(ValueError):
        config_from_par_text(base % 16)


def test_small_values_from_par_file(tmp_path):
    """fix_small_values, small_values_method and small_values_daverage of
    &methodlist reach the configuration (src/mod_small_values.t:9-12)."""
    from amrvac_b200.config import config_from_par
    f = tmp_path / "sv.par"
    f.write_text("""
 &methodlist
        time_stepper = 'threestep'
        flux_scheme = 20*'hllc'
        limiter = 20*'cada3'
        fix_small_values = .true.
        small_values_method = 'average'
        small_values_daverage = 2
        small_density = 1.d-6
        small_pressure = 1.d-7
 /
 &meshlist
        domain_nx1=32
        domain_nx2=32
 /
 &hd_list
 /
""")
    rc = config_from_par([str(f)])
    c = rc.cfg
    assert c.fix_small_values == 1 and c.small_values_method == 2 and c.small_values_daverage == 2
    assert c.small_density == 1e-6 and c.small_pressure == 1e-7


def test_stage_variant_entry_points_check_their_arguments(lib):
    """The launch-shape entry points refuse a null context (no device
    needed)."""
    v = [ctypes.c_int() for _ in range(5)]
    assert lib.amrvac_gpu_set_stage_variant(None, 0) < 0
    assert lib.amrvac_gpu_stage_variant(None, *[ctypes.byref(x) for x in v]) < 0
    assert lib.amrvac_gpu_set_zchunk(None, 0) < 0


def test_wait_probe_checks_its_arguments(lib):
    """The bounded-wait diagnostic refuses a null result and spin counts
    outside 1 .. 4194304 before any device work."""
    f = ctypes.c_uint32(0)
    assert lib.amrvac_gpu_wait_probe(100, None) < 0
    assert lib.amrvac_gpu_wait_probe(0, ctypes.byref(f)) < 0
    assert lib.amrvac_gpu_wait_probe((1 << 22) + 1, ctypes.byref(f)) < 0


def test_step_with_caller_stage_buffers_checks_its_arguments(lib):
    """amrvac_gpu_step_dt_states refuses a null context before it touches a
    buffer (no device needed)."""
    assert lib.amrvac_gpu_step_dt_states(None, 1.0, None, None, None, None) < 0


def test_par_namelist_parser():
    from amrvac_b200 import parse_namelists
    text = """
 &methodlist
        time_stepper  = 'threestep'
        flux_scheme =    20*'hlld'
        limiter=  20*'cada3'
        typeboundspeed  = 'cmaxmean'
 /
 &meshlist
        domain_nx1    = 128
        xprobmin1     = -1.d0
        w_refine_weight(1)=0.5d0
 /
 &paramlist
        courantpar = 0.9
 /
"""
    nl = parse_namelists(text)
    assert nl["methodlist"]["flux_scheme"] == ["hlld"] * 20
    assert nl["methodlist"]["time_stepper"] == "threestep"
    assert nl["meshlist"]["domain_nx1"] == 128
    assert nl["meshlist"]["xprobmin1"] == -1.0
    assert nl["meshlist"]["w_refine_weight"] == {1: 0.5}
    assert nl["paramlist"]["courantpar"] == 0.9


def test_config_from_par(tmp_path):
    from amrvac_b200 import config_from_par
    p = tmp_path / "kh.par"
    p.write_text("""
 &stoplist
    time_max = 1.0
 /
 &methodlist
    time_stepper = 'threestep'
    flux_scheme = 20*'hllc'
    limiter = 20*'vanleer'
 /
 &boundlist
    typeboundary_min1 = 4*'periodic'
    typeboundary_max1 = 4*'periodic'
    typeboundary_min2 = 4*'periodic'
    typeboundary_max2 = 4*'periodic'
 /
 &meshlist
    domain_nx1 = 256
    domain_nx2 = 256
    xprobmin2 = -0.5
    xprobmax2 = 0.5
 /
 &hd_list
    hd_gamma = 1.4
 /
""")
    rc = config_from_par([str(p)])
    assert rc.physics == "hd" and rc.domain_nx == [256, 256]
    assert rc.cfg.flux_scheme == 3 and rc.cfg.limiter == 5 and rc.cfg.gamma == 1.4
    assert rc.cfg.time_stepper == 3 and rc.xprobmin == [0.0, -0.5]


def test_time_integrators_are_checked():
    """twostep is Predictor_Corrector by default (the reference's default) or
    ssprk2 on request; TVDLF's Hancock predictor is FP64 only, so the mixed
    form of that pair is refused at creation (which needs no device: the
    check comes first)."""
    from amrvac_b200 import _lib, make_cfg
    lib = _lib.load()
    import ctypes
    h = ctypes.c_void_p()
    bad = make_cfg(physics="hd", ndim=2, flux_scheme="tvdlf", time_stepper="twostep", precision="mixed")
    assert lib.amrvac_gpu_create(ctypes.byref(bad), ctypes.byref(h)) == _lib.E_UNSUPPORTED
    bad = make_cfg(physics="hd", ndim=2, flux_scheme="hll", time_stepper="threestep", time_integrator="rk4")
    assert lib.amrvac_gpu_create(ctypes.byref(bad), ctypes.byref(h)) == _lib.E_UNSUPPORTED
    ok = make_cfg(physics="hd", ndim=2, flux_scheme="hll", time_stepper="twostep")
    assert ok.time_stepper == 2 and ok.time_integrator == 0
    assert make_cfg(physics="hd", ndim=2, time_stepper="twostep", time_integrator="ssprk2").time_integrator == 2
    assert make_cfg(physics="hd", ndim=2, time_stepper="fivestep").time_stepper == 5
    bad = make_cfg(physics="hd", ndim=2, flux_scheme="hll", time_stepper="fivestep", ssprk_order=4)
    assert lib.amrvac_gpu_create(ctypes.byref(bad), ctypes.byref(h)) == _lib.E_ARG


def test_mp5_needs_three_ghost_cells_and_fp64(lib):
    """MP5 (limiter 13) is taken with nghostcells >= 3 (make_cfg's default for
    it) in FP64; two ghost cells or the mixed form are refused before any
    device call."""
    from amrvac_b200 import make_cfg, _lib
    h = ctypes.c_void_p()
    assert make_cfg(physics="hd", ndim=2, limiter="mp5").nghostcells == 3
    assert make_cfg(physics="hd", ndim=2).nghostcells == 2
    assert make_cfg(physics="hd", ndim=2, limiter="wenozp5").nghostcells == 3
    bad = make_cfg(physics="hd", ndim=2, flux_scheme="hll", limiter="mp5", nghostcells=2)
    assert lib.amrvac_gpu_create(ctypes.byref(bad), ctypes.byref(h)) == _lib.E_ARG
    bad = make_cfg(physics="hd", ndim=2, flux_scheme="hll", limiter="mp5", precision="mixed")
    assert lib.amrvac_gpu_create(ctypes.byref(bad), ctypes.byref(h)) == _lib.E_UNSUPPORTED


def test_config_from_par_reads_the_method_options(tmp_path):
    """methodlist options of the reconstructions, steppers and splitting:
    twostep TVD-MUSCL dimensionally split; fivestep with MP5 (three ghost
    cells by default, as the reference sets them); schmid2 radii."""
    from amrvac_b200 import config_from_par
    from amrvac_b200 import _lib
    common = """
 &meshlist
        domain_nx1 = 64
        domain_nx2 = 64
 /
 &paramlist
        courantpar = 0.9
 /
"""
    p = tmp_path / "a.par"
    p.write_text(""" &methodlist
        time_stepper = 'twostep'
        flux_scheme = 20*'tvdmu'
        limiter = 20*'albada'
        dimsplit = .true.
        typeboundspeed = 'cmaxmean'
 /
""" + common)
    c = config_from_par([str(p)]).cfg
    assert (c.time_stepper, c.flux_scheme, c.limiter, c.dimsplit) == (2, _lib.FS["tvdmu"], 6, 1)
    assert c.typeboundspeed == 2 and c.nghostcells == 2
    p.write_text(""" &methodlist
        time_stepper = 'fivestep'
        flux_scheme = 20*'hll'
        limiter = 20*'mp5'
        dimsplit = .true.
        typedimsplit = 'xy'
 /
""" + common)
    c = config_from_par([str(p)]).cfg
    assert (c.time_stepper, c.limiter, c.nghostcells, c.dimsplit) == (5, 13, 3, 2)
    p.write_text(""" &methodlist
        limiter = 20*'schmid2'
        schmid_rad1 = 2.5d0
        schmid_rad2 = 0.5d0
 /
""" + common)
    c = config_from_par([str(p)]).cfg
    assert c.limiter == 10 and list(c.schmid_rad) == [2.5, 0.5, 1.0] and c.schmid_global == 0
    from amrvac_b200 import make_cfg
    assert make_cfg(limiter="schmid1").schmid_global == 1


def test_product_fails_loudly_without_the_library(tmp_path):
    """With the CUDA library absent there is no fallback: creating a context
    raises ImportError naming the missing library (fresh process)."""
    import subprocess
    import sys
    env = dict(os.environ, AMRVAC_GPU_LIB=str(tmp_path / "missing" / "libamrvac_gpu.so"))
    code = ("from amrvac_b200 import Context, make_cfg\n"
            "Context(make_cfg(physics='hd', ndim=2))\n")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode != 0
    assert "ImportError" in r.stderr and "There is no CPU fallback" in r.stderr
