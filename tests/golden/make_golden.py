"""Copy the reference's golden regression logs for the finite-volume path.

Run once in a checkout that has the reference repository next to it:

    python tests/golden/make_golden.py /path/to/amrvac

The logs are the reference's own correct_output fixtures: the only
uniform-grid (refine_max_level=1) regression tests on the HLL/HLLD path,
tests/mhd/field_loop_2.5D/correct_output/fl_2d_3step_{hlld,hll}_cada.log, and
the periodic multi-level tests on the same schemes,
tests/mhd/Orszag_Tang_2D/correct_output/ot_2d_3step_{hlld,hll}_cada.log and
tests/hd/Kelvin_Helmholtz_2D/correct_output/kh_2d_3step_hll_cada.log, and the
fourstep variants (rk4 with HLL and woodward, ssprk4 with HLLC and koren)
ot_2d_4step_hll_mc.log, kh_2d_4step_hll_mc.log, kh_2d_4step_hllc_ko.log and
(RK4, TVDLF, cada3) ot_2d_rk4_tvdlf_cada.log, kh_2d_rk4_tvdlf_cada.log, and
the twostep Predictor_Corrector variant (MUSCL-Hancock predictor, TVDLF,
minmod) ot_2d_2step_tvdlf_mm.log, and MHD HLLC (SSPRK(4,3), koren, Linde)
ot_2d_4step_hllc_ko.log, and MHD TVD-MUSCL (dimensionally split, albada)
ot_2d_2step_tvdmu_al.log; and the 2-D blast wave with cont
boundaries, tests/hd/blast_wave_Cartesian_2D/correct_output/
bw_2d_{3step_hll_cada,4step_hll_mc,4step_hllc_ko,rk4_tvdlf_cada,
2step_tvdlf_mm,2step_tvdmu_al}.log (the last with TVD-MUSCL, dimensionally
split); the 3-D MHD blast wave (8^3 blocks), the 2-D Riemann problem (12^2
blocks) and the 3-D MHD Kelvin-Helmholtz jet (10^3 blocks) in the schemes
listed below.
They are copied verbatim so the parity tests can run where the reference
repository is absent.
"""
import os
import shutil
import sys

LOGS = [
    "tests/mhd/field_loop_2.5D/correct_output/fl_2d_3step_hlld_cada.log",
    "tests/mhd/field_loop_2.5D/correct_output/fl_2d_3step_hll_cada.log",
    # multi-level (refine_max_level = 3, Löhner, regrid every step), periodic
    "tests/mhd/Orszag_Tang_2D/correct_output/ot_2d_3step_hlld_cada.log",
    "tests/mhd/Orszag_Tang_2D/correct_output/ot_2d_3step_hll_cada.log",
    "tests/hd/Kelvin_Helmholtz_2D/correct_output/kh_2d_3step_hll_cada.log",
    "tests/mhd/Orszag_Tang_2D/correct_output/ot_2d_4step_hll_mc.log",
    "tests/hd/Kelvin_Helmholtz_2D/correct_output/kh_2d_4step_hll_mc.log",
    "tests/hd/Kelvin_Helmholtz_2D/correct_output/kh_2d_4step_hllc_ko.log",
    "tests/mhd/Orszag_Tang_2D/correct_output/ot_2d_rk4_tvdlf_cada.log",
    "tests/hd/Kelvin_Helmholtz_2D/correct_output/kh_2d_rk4_tvdlf_cada.log",
    "tests/mhd/Orszag_Tang_2D/correct_output/ot_2d_2step_tvdlf_mm.log",
    "tests/mhd/Orszag_Tang_2D/correct_output/ot_2d_4step_hllc_ko.log",
    "tests/mhd/Orszag_Tang_2D/correct_output/ot_2d_2step_tvdmu_al.log",
    # multi-level with cont boundaries
    "tests/hd/blast_wave_Cartesian_2D/correct_output/bw_2d_3step_hll_cada.log",
    "tests/hd/blast_wave_Cartesian_2D/correct_output/bw_2d_4step_hll_mc.log",
    "tests/hd/blast_wave_Cartesian_2D/correct_output/bw_2d_4step_hllc_ko.log",
    "tests/hd/blast_wave_Cartesian_2D/correct_output/bw_2d_rk4_tvdlf_cada.log",
    "tests/hd/blast_wave_Cartesian_2D/correct_output/bw_2d_2step_tvdlf_mm.log",
    "tests/hd/blast_wave_Cartesian_2D/correct_output/bw_2d_2step_tvdmu_al.log",
    # 3-D multi-level with 8^3 blocks (block_nx 8), cont boundaries
    "tests/mhd/blast_wave_Cartesian_3D/correct_output/bw_3d_3step_hlld_cada.log",
    "tests/mhd/blast_wave_Cartesian_3D/correct_output/bw_3d_3step_hll_cada.log",
    "tests/mhd/blast_wave_Cartesian_3D/correct_output/bw_3d_3step_hll_ko.log",
    "tests/mhd/blast_wave_Cartesian_3D/correct_output/bw_3d_4step_hll_mc.log",
    "tests/mhd/blast_wave_Cartesian_3D/correct_output/bw_3d_4step_hllc_ko.log",
    "tests/mhd/blast_wave_Cartesian_3D/correct_output/bw_3d_rk4_tvdlf_cada.log",
    "tests/mhd/blast_wave_Cartesian_3D/correct_output/bw_3d_2step_tvdlf_mm.log",
    # 2-D HD with 12^2 blocks (block_nx 12), cont boundaries
    "tests/hd/Riemann_2D/correct_output/rm_2d_3step_hll_cada.log",
    "tests/hd/Riemann_2D/correct_output/rm_2d_4step_hll_mc.log",
    "tests/hd/Riemann_2D/correct_output/rm_2d_4step_hllc_ko.log",
    "tests/hd/Riemann_2D/correct_output/rm_2d_rk4_tvdlf_cada.log",
    "tests/hd/Riemann_2D/correct_output/rm_2d_2step_tvdlf_mm.log",
    "tests/hd/Riemann_2D/correct_output/rm_2d_2step_tvdmu_al.log",
    # 3-D MHD with 10^3 blocks (block_nx 10), periodic x, cont y and z
    "tests/mhd/Kelvin_Helmholtz_3D/correct_output/kh_3D_3step_hll_cada.log",
    "tests/mhd/Kelvin_Helmholtz_3D/correct_output/kh_3D_3step_hlld_cada.log",
    "tests/mhd/Kelvin_Helmholtz_3D/correct_output/kh_3D_4step_hll_mc.log",
    "tests/mhd/Kelvin_Helmholtz_3D/correct_output/kh_3D_4step_hllc_ko.log",
    "tests/mhd/Kelvin_Helmholtz_3D/correct_output/kh_3D_rk4_tvdlf_cada.log",
    "tests/mhd/Kelvin_Helmholtz_3D/correct_output/kh_3D_2step_tvdlf_mm.log",
    "tests/mhd/Kelvin_Helmholtz_3D/correct_output/kh_3D_2step_tvdmu_al.log",
]


def main(ref_root: str) -> None:
    here = os.path.dirname(os.path.abspath(__file__))
    for rel in LOGS:
        src = os.path.join(ref_root, rel)
        dst = os.path.join(here, os.path.basename(rel))
        shutil.copyfile(src, dst)
        print("wrote", dst)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("AMRVAC_REFERENCE")
    if not ref:
        sys.exit(f"usage: python {os.path.basename(__file__)} <MPI-AMRVAC source root> "
                 "(or set AMRVAC_REFERENCE)")
    main(ref)
