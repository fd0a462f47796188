"""Problem set-ups used by the tests, as reference-format input text.

Each set-up names one of the reference's problem generators (src/pgen.hpp:269-307) so that
the oracle produces the initial state itself; the device mesh is then loaded with exactly
that state.
"""

ORSZAG_TANG = """
[mesh]
nx1 = {n}
nx2 = {n}
nx3 = 1
x1min = 0.0
x1max = 1.0
x2min = 0.0
x2max = 1.0
[time]
integrator = rk3
cfl = 0.4
tlim = 0.5
[mhd]
gamma = 1.6666666666666667
reconstruct = ppm
rsolver = hlld
[problem]
name = orszag_tang
"""

BLAST_3D = """
[mesh]
nx1 = {n}
nx2 = {n}
nx3 = {n}
x1min = -0.5
x1max = 0.5
x2min = -0.5
x2max = 0.5
x3min = -0.5
x3max = 0.5
[time]
integrator = rk3
cfl = 0.4
tlim = 0.2
[mhd]
gamma = 1.6666666666666667
reconstruct = ppm
rsolver = hlld
[problem]
name = blast
pres_in = 10.0
pres_out = 0.1
radius = 0.1
b0 = 1.0
angle = 45.0
"""

CPAW = """
[mesh]
nx1 = {n1}
nx2 = {n2}
nx3 = {n3}
x1min = 0.0
x1max = {l1}
x2min = 0.0
x2max = {l2}
x3min = 0.0
x3max = {l3}
[time]
integrator = rk3
cfl = 0.4
tlim = 1.0
[mhd]
gamma = 1.6666666666666667
reconstruct = wenoz
rsolver = hlld
[problem]
name = cpaw
dens = 1.0
pres = 0.1
b_par = 1.0
amp = 0.1
lambda = 1.0
angle = {angle}
"""

SHOCK_TUBE = """
[mesh]
nx1 = {n}
nx2 = 1
nx3 = 1
x1min = -0.5
x1max = 0.5
bc_x1 = outflow
[time]
integrator = rk3
cfl = 0.4
tlim = 0.1
[mhd]
gamma = 2.0
reconstruct = ppm
rsolver = hlld
[problem]
name = shock_tube
"""

FIELD_LOOP = """
[mesh]
nx1 = {n}
nx2 = {n}
nx3 = {n3}
x1min = -0.5
x1max = 0.5
x2min = -0.5
x2max = 0.5
x3min = -0.5
x3max = 0.5
[time]
integrator = rk3
cfl = 0.4
tlim = 1.0
[mhd]
reconstruct = ppmx
rsolver = hlld
[problem]
name = field_loop
vz = 0.3
"""


def ot(n=32):
    return ORSZAG_TANG.format(n=n)


def blast(n=16):
    return BLAST_3D.format(n=n)


def cpaw1d(n=32):
    return CPAW.format(n1=n, n2=1, n3=1, l1=1.0, l2=1.0, l3=1.0, angle=0.0)


def cpaw2d(n=32):
    return CPAW.format(n1=n, n2=n, n3=1, l1=1.4142135623730951, l2=1.4142135623730951, l3=1.0, angle=45.0)


def cpaw3d_extruded(n=16, nz=8):
    return CPAW.format(n1=n, n2=n, n3=nz, l1=1.4142135623730951, l2=1.4142135623730951,
                       l3=1.4142135623730951 * nz / n, angle=45.0)


def shock_tube(n=64):
    return SHOCK_TUBE.format(n=n)


def field_loop(n=16, n3=1):
    return FIELD_LOOP.format(n=n, n3=n3)


# Sinusoidal decay set-up of the reference's physics tests (diffusion_test generator,
# src/pgen.hpp:235-266); the coefficient and the perturbed variable come as overrides.
DIFFUSION = """
[mesh]
nx1 = {n1}
nx2 = {n2}
nx3 = {n3}
[time]
integrator = rk3
cfl = 0.3
tlim = 0.5
[mhd]
reconstruct = plm
[problem]
name = diffusion_test
var = {var}
axis = {axis}
amp = 1.0e-3
"""


def diffusion(var="b", axis=1, n=64, n_other=8):
    dims = [1, 1, 1]
    for a in range(axis):
        dims[a] = n_other
    dims[axis - 1] = n
    return DIFFUSION.format(n1=dims[0], n2=dims[1], n3=dims[2], var=var, axis=axis)
