"""Golden files for the reference's file formats.

Run in a container where the reference project is importable (nothing at test
time imports it):

    python tests/golden/make_golden_io.py --reference /path/to/DNS-Supercritical-IBM

1. Field snapshot (src/mod_io.f90:7-149): tests/golden/field_5x3x4.dat written
   with the reference's own Python writer (misc/reinterp/tester_mk_ini_data_bin.py:54-61,
   the format cfd_read_arr reads) and tests/golden/field_5x3x4.npz with the
   values; the file is checked with the reference's reader
   (CFD_Folder.import_array_bin, :174-183).

2. Geometry files of a case (the geom_data folder that src/pycode/calc_bands.py
   writes and src/inc_set_alloc_arrays.f90:54-59 / src/inc_set_read_params.f90
   read): tests/golden/geom_12/{P_band_abc, P_band_abc_00, inv_dy_p,
   dPdy_ddy_lh}.dat and base_params.txt for a 12-cell tanh grid.  The bands come
   from calc_bands.mk_P_abc (:181-201) and every file is written by
   calc_bands.writer (:26-31) with the row format of its mk_geom_vars_write
   (:358-364: first line the row count, then the row values joined by spaces,
   each value as Python's str of the float).  inv_dy_p and dPdy_ddy_lh follow
   :274 and :336-343; base_params.txt follows the line layout of :247-266.
   tests/golden/geom_12.npz holds the same values as float64 arrays.
"""
import argparse
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def make_field(ref_root):
    sys.path.insert(0, os.path.join(ref_root, "misc", "reinterp"))
    import tester_mk_ini_data_bin as ref  # the reference's binary writer and reader
    A = np.random.default_rng(21).normal(size=(5, 3, 4))
    A[0, 0, 0] = np.pi  # an exactly known first value
    path = os.path.join(HERE, "field_5x3x4.dat")
    ref.writer_bin(path, A, [5, 3, 4])
    np.savez(os.path.join(HERE, "field_5x3x4.npz"), A=A)
    back = ref.CFD_Folder.import_array_bin(path)
    assert np.array_equal(back, A)
    print("wrote", path, os.path.getsize(path), "bytes")


def make_geom(ref_root):
    sys.path.insert(0, os.path.join(ref_root, "src", "pycode"))
    import calc_bands as cb  # the reference's band generator and text writer
    ny, nx, nz = 12, 16, 8
    yu = [float(1.0 + math.tanh(2.0 * (2.0 * j / ny - 1.0)) / math.tanh(2.0)) for j in range(ny + 1)]
    yp = [(yu[i] + yu[i + 1]) / 2 for i in range(ny)]
    yp_ext = [yu[0]] + yp + [yu[-1]]
    result = {
        "inv_dy_p": [1. / (yu[i + 1] - yu[i]) for i in range(ny)],
        "P_band_abc": cb.mk_P_abc(yp_ext, is_dirich_first=False),
        "P_band_abc_00": cb.mk_P_abc(yp_ext, is_dirich_first=True),
        "dPdy_ddy_lh": [],
    }
    for i in range(ny + 1):
        if i in (0, ny):
            result["dPdy_ddy_lh"].append([0., 0.])
        else:
            dy = yp[i] - yp[i - 1]
            result["dPdy_ddy_lh"].append([-1 / dy, 1 / dy])
    folder = os.path.join(HERE, "geom_12")
    for key, A in result.items():
        if type(A[0]) in [float, int]:
            A = [[x] for x in A]
        cb.writer(os.path.join(folder, f"{key}.dat"), [str(len(A)), *[" ".join(map(str, row)) for row in A]])
    Lx, Lz, dtmax = 2 * math.pi, math.pi, 0.25
    base = [f"{nx} {nz} {ny} ! nx nz ny_total",
            "0 0 ! use_rough_surf use_rough_surf_quady",
            f"100 {dtmax} ! nstep dtmax",
            f"{Lx / nx} {Lz / nz} ! dx dz",
            "0.01 0.01 ! nu cond",
            "1.0 0.0 0.0 ! Sf_x Sf_z Sq",
            "0.0 0.0 0.0 ! Gb_x Gb_z Gb_y",
            "1 1 1 0 ! avg_iter_start avg_nraw avg_freq avg_bin_nbins",
            "1 -1 ! snap_iter_start snap_freq",
            "10 ! bulk_nprint",
            "-1 -1 -1 ! filtering_steps filtering_first filtering_nstop",
            "0.0 0.0 0.0 1.0 ! wall_BC_U/V/W/T_bot",
            "0.5 0.0 -0.25 1.0 ! wall_BC_U/V/W/T_top",
            "1 ! use_incompressible"]
    cb.writer(os.path.join(folder, "base_params.txt"), base)
    np.savez(os.path.join(HERE, "geom_12.npz"), yu=np.array(yu),
             P_band_abc=np.array(result["P_band_abc"]), P_band_abc_00=np.array(result["P_band_abc_00"]),
             inv_dy_p=np.array(result["inv_dy_p"]), dPdy_ddy_lh=np.array(result["dPdy_ddy_lh"]),
             grid=np.array([nx, nz, ny]), dxdz=np.array([Lx / nx, Lz / nz]), dtmax=np.array(dtmax),
             walls=np.array([0.0, 0.0, 0.0, 0.5, 0.0, -0.25]))
    print("wrote", folder)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="root of the reference project checkout")
    args = ap.parse_args()
    make_field(args.reference)
    make_geom(args.reference)


if __name__ == "__main__":
    main()
