"""Writes the golden fixtures of tests/test_golden.py from the reference itself: each case's
input file is run by the reference's own kernels compiled in place (oracle/_ref/libchqref.so,
built by `make -C oracle` from the reference sources) and the initial and final states, the
clock and the history sums are stored in tests/golden/<case>.npz.

    python tests/golden/make_golden.py [case ...]   # needs oracle/_ref (the reference sources)

The fixtures let the parity tests run where the reference is not available."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from tests import cases  # noqa: E402

FIELDS = ("u0", "b1f0", "b2f0", "b3f0")

# name: (input text, overrides, cycles)
CASES = {
    "ot2d_16_ppm_hlld": (cases.ot(16), [], 6),
    "blast3d_12_strong_fofc": (cases.blast(12), ["problem.pres_in=1e4", "problem.pres_out=1e-3", "time.cfl=0.5"], 5),
    "cpaw1d_32_wenoz_hlld": (cases.cpaw1d(32), [], 8),
    "loop3d_8_ppmx_lhlld_char": (cases.field_loop(8, 4), ["mhd.rsolver=lhlld", "mhd.characteristic=true"], 4),
    "ot2d_16_diffusion": (cases.ot(16), ["diffusion.nu=2e-3", "diffusion.kappa=2e-3", "diffusion.eta=1e-3"], 5),
    "ot2d_16_gravity_cooling": (cases.ot(16), ["gravity.uniform=true", "gravity.g1=0.5", "gravity.g2=-0.25",
                                                "cooling.enabled=true", "cooling.lambda0=0.5"], 5),
    "shock1d_64_plm_hlle_rk2": (cases.shock_tube(64), ["mhd.reconstruct=plm", "mhd.rsolver=hlle",
                                                       "time.integrator=rk2"], 10),
    # RKL2 resistivity with five super-time-stepping stages per cycle
    "ot2d_16_rkl2_eta": (cases.ot(16), ["diffusion.eta=0.2", "diffusion.sts=true"], 5),
    # softened point mass on the strong blast, with first-order flux corrections
    "blast3d_12_point_mass_fofc": (cases.blast(12), ["gravity.point_mass=true", "gravity.gm=0.05", "gravity.x0=0.05",
                                                     "gravity.y0=-0.1", "gravity.z0=0.02", "gravity.rsoft=0.05",
                                                     "problem.pres_in=1e4", "problem.pres_out=1e-3",
                                                     "time.cfl=0.5"], 4),
}


def main():
    from oracle.refsim import RefSim, available
    if not available():
        raise SystemExit("oracle/_ref is not built (make -C oracle with the reference sources present)")
    only = set(sys.argv[1:])
    for name, (text, ov, ncyc) in CASES.items():
        if only and name not in only:
            continue
        ref = RefSim(text, list(ov))
        data = {"text": np.array(text), "overrides": np.array(ov if ov else [""]), "cycles": np.array(ncyc)}
        for f in FIELDS:
            data["in_" + f] = ref.get(f)
        ref.cycles(ncyc)
        for f in FIELDS:
            data["out_" + f] = ref.get(f)
        data["time"] = np.array(ref.time)
        data["cycle"] = np.array(ref.cycle)
        data["fofc"] = np.array(ref.fofc_count)
        data["history"] = np.array(ref.history())
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **data)
        ref.close()
        print(name, int(data["cycle"]), "cycles, t =", float(data["time"]), "fofc", int(data["fofc"]))


if __name__ == "__main__":
    main()
