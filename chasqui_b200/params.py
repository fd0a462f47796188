"""Reference-compatible parameter handling.

`Params` reads the reference's INI dialect (``[block]``, ``key = value  # comment``) and its
``block.key=value`` command-line overrides with the same semantics as src/params.hpp:17-92:
later keys win, ``get_or_add_*`` records the default so that the effective table echoes every
key used, booleans accept true/1/yes. `config_from_params` reads the same keys with the same
defaults as src/main.cpp:113-185 and returns the fields of ``chq_config`` plus the driver
keys (tlim, nlim, ndiag, problem, outputs).
"""
from __future__ import annotations


class ParamError(RuntimeError):
    pass


class Params:
    def __init__(self):
        self._t: dict[str, str] = {}

    # src/params.hpp:19-36
    def read_file(self, fname: str) -> "Params":
        try:
            text = open(fname).read()
        except OSError as e:
            raise ParamError(f"cannot open input file: {fname}") from e
        return self.read_text(text)

    def read_text(self, text: str) -> "Params":
        block = ""
        for line in text.splitlines():
            h = line.find("#")
            if h >= 0:
                line = line[:h]
            line = line.strip()
            if not line:
                continue
            if line[0] == "[" and line[-1] == "]":
                block = line[1:-1].strip()
                continue
            eq = line.find("=")
            if eq < 0:
                continue
            self._t[block + "." + line[:eq].strip()] = line[eq + 1:].strip()
        return self

    # src/params.hpp:38-43
    def override(self, arg: str) -> None:
        eq = arg.find("=")
        if eq < 0:
            raise ParamError("bad override: " + arg)
        self._t[arg[:eq].strip()] = arg[eq + 1:].strip()

    def has(self, b: str, k: str) -> bool:
        return f"{b}.{k}" in self._t

    def get_string(self, b: str, k: str) -> str:
        key = f"{b}.{k}"
        if key not in self._t:
            raise ParamError("missing parameter " + key)
        return self._t[key]

    def get_or_add_string(self, b: str, k: str, d: str) -> str:
        return self._t.setdefault(f"{b}.{k}", d)

    def get_real(self, b: str, k: str) -> float:
        return float(self.get_string(b, k))

    def get_or_add_real(self, b: str, k: str, d: float) -> float:
        key = f"{b}.{k}"
        if key not in self._t:
            self._t[key] = repr(float(d))
        return float(self._t[key])

    def get_int(self, b: str, k: str) -> int:
        return int(self.get_string(b, k))

    def get_or_add_int(self, b: str, k: str, d: int) -> int:
        key = f"{b}.{k}"
        if key not in self._t:
            self._t[key] = str(int(d))
        return int(self._t[key])

    def get_or_add_bool(self, b: str, k: str, d: bool) -> bool:
        key = f"{b}.{k}"
        if key not in self._t:
            self._t[key] = "true" if d else "false"
        return self._t[key].lower() in ("true", "1", "yes")

    def items(self):
        return sorted(self._t.items())

    def text(self) -> str:
        """The table as an input file (block order sorted, like Params::Print)."""
        out, last = [], None
        for key, v in self.items():
            b, k = key.split(".", 1)
            if b != last:
                out.append(f"[{b}]")
                last = b
            out.append(f"{k} = {v}")
        return "\n".join(out) + "\n"


RECON = {"dc": 0, "plm": 1, "ppm": 2, "wenoz": 3, "ppmx": 4}
RSOLVER = {"hlle": 0, "hlld": 1, "lhlld": 2}
INTEGRATOR = {"rk1": 1, "rk2": 2, "rk3": 3, "rk4": 4, "ssprk43": 4}
BC = {"periodic": 0, "outflow": 1, "reflect": 2}


def config_from_params(pin: Params) -> dict:
    """Keys and defaults of src/main.cpp:113-185, as chq_config fields + driver settings."""
    c: dict = {}
    r = pin.get_or_add_string("mhd", "reconstruct", "ppm")
    if r not in RECON:
        raise ParamError("unknown reconstruct: " + r)
    c["recon"] = RECON[r]
    s = pin.get_or_add_string("mhd", "rsolver", "hlld")
    if s not in RSOLVER:
        raise ParamError("unknown rsolver: " + s)
    c["rsolver"] = RSOLVER[s]
    c["characteristic"] = int(pin.get_or_add_bool("mhd", "characteristic", False))
    c["lhlld_phi"] = pin.get_or_add_real("mhd", "lhlld_phi", -1.0)
    c["dual_energy"] = int(pin.get_or_add_bool("mhd", "dual_energy", False))
    c["de_eta"] = pin.get_or_add_real("mhd", "de_eta", 1.0e-3)
    t = pin.get_or_add_string("time", "integrator", "rk3")
    if t not in INTEGRATOR:
        raise ParamError("unknown integrator: " + t)
    c["integrator"] = INTEGRATOR[t]
    c["low_mach"] = int(pin.get_or_add_bool("mhd", "low_mach", False))
    c["flatten"] = int(pin.get_or_add_bool("mhd", "flatten", True))
    c["cfl"] = pin.get_or_add_real("time", "cfl", 0.3)
    c["gamma"] = pin.get_or_add_real("mhd", "gamma", 5.0 / 3.0)
    c["dfloor"] = pin.get_or_add_real("mhd", "dfloor", 1.0e-10)
    c["pfloor"] = pin.get_or_add_real("mhd", "pfloor", 1.0e-12)
    for q, key in ((1, "bc_x1"), (2, "bc_x2"), (3, "bc_x3")):
        b = pin.get_or_add_string("mesh", key, "periodic")
        if b not in BC:
            raise ParamError("unknown boundary condition: " + b)
        c[f"bc{q}"] = BC[b]
    c["fofc"] = int(pin.get_or_add_bool("mhd", "fofc", True))
    c["flux_limiter"] = int(pin.get_or_add_bool("mhd", "flux_limiter", False))
    c["sts"] = int(pin.get_or_add_bool("diffusion", "sts", False))
    c["nu"] = pin.get_or_add_real("diffusion", "nu", 0.0)
    c["kappa"] = pin.get_or_add_real("diffusion", "kappa", 0.0)
    c["eta"] = pin.get_or_add_real("diffusion", "eta", 0.0)
    c["gravity_uniform"] = int(pin.get_or_add_bool("gravity", "uniform", False))
    c["g1"] = pin.get_or_add_real("gravity", "g1", 0.0)
    c["g2"] = pin.get_or_add_real("gravity", "g2", 0.0)
    c["g3"] = pin.get_or_add_real("gravity", "g3", 0.0)
    c["gravity_point"] = int(pin.get_or_add_bool("gravity", "point_mass", False))
    c["gm"] = pin.get_or_add_real("gravity", "gm", 0.0)
    c["gx0"] = pin.get_or_add_real("gravity", "x0", 0.0)
    c["gy0"] = pin.get_or_add_real("gravity", "y0", 0.0)
    c["gz0"] = pin.get_or_add_real("gravity", "z0", 0.0)
    c["rsoft"] = pin.get_or_add_real("gravity", "rsoft", 0.0)
    c["cooling"] = int(pin.get_or_add_bool("cooling", "enabled", False))
    c["lambda0"] = pin.get_or_add_real("cooling", "lambda0", 0.0)
    c["cool_alpha"] = pin.get_or_add_real("cooling", "alpha", 1.0)
    c["tfloor"] = pin.get_or_add_real("cooling", "tfloor", 0.0)
    c["nx1"] = pin.get_int("mesh", "nx1")
    c["nx2"] = pin.get_or_add_int("mesh", "nx2", 1)
    c["nx3"] = pin.get_or_add_int("mesh", "nx3", 1)
    ng_min = 3 if r in ("ppm", "ppmx", "wenoz") else 2
    c["nghost"] = pin.get_or_add_int("mesh", "nghost", ng_min)
    if c["nghost"] < ng_min:
        raise ParamError("nghost too small for the reconstruction method")
    for ax in ("x1", "x2", "x3"):
        c[f"{ax}min"] = pin.get_or_add_real("mesh", f"{ax}min", 0.0)
        c[f"{ax}max"] = pin.get_or_add_real("mesh", f"{ax}max", 1.0)
    c["tlim"] = pin.get_or_add_real("time", "tlim", 1.0)
    c["nlim"] = pin.get_or_add_int("time", "nlim", -1)
    prec = pin.get_or_add_string("mhd", "precision", "fp64")
    if prec not in ("fp64", "mixed"):
        raise ParamError("unknown precision: " + prec)
    c["precision"] = 0 if prec == "fp64" else 1
    return c
