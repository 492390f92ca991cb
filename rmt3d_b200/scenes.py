"""Synthetic workloads of this path as reference .cfg files.

Each builder returns the text of a .cfg file in the reference's keyword
format (Sim/sim_params.cc:10-410), so the same file drives both this
implementation and the reference's own run_sim.  The lid-driven cavity and
the spheres are defined entirely by these parameters; nothing is read from a
dataset.
"""
import math
import random

_WALLS_LID = """bc_xl 1 1 1 0 0 0
bc_xh 1 1 1 0 0 0
bc_yl 1 1 1 0 0 0
bc_yh 1 1 1 0 0 0
bc_zl 1 1 1 0 0 0
bc_zh 1 1 1 {lid} 0 0
"""

_HEAD = """suppress 1
dump_code 0
ntracers 0
frames {frames}
stop_short {steps}
sys_size {n} {n} {n}
xyz_bounds 0 1 0 1 0 1
dt 10
T {T}
sim_type objects
fmu {mu}
"""


def cavity(n=32, steps=64, mu=0.01, lid=1.0, frames=100000, T=None):
    """Lid-driven cavity, unit cube, no-slip walls, lid u=(lid,0,0) at z=1."""
    if T is None:
        T = frames
    return _HEAD.format(frames=frames, steps=steps, n=n, T=T, mu=mu) + _WALLS_LID.format(lid=lid)


def cavity_sphere(n=64, steps=200, mu=0.01, G=1.0, rho=1.0, radius=0.2, centre=(0.5, 0.5, 0.5),
                  wt_n=1.5, nlayers=5, frames=100000, T=None):
    """Lid-driven cavity holding one neo-Hookean sphere with the identity map."""
    s = cavity(n, steps, mu, 1.0, frames, T)
    s += "wt_n %g\nnlayers %d\nn_obj 1\nobject_list 0 0\n" % (wt_n, nlayers)
    s += "basic_specs 0 %r %r %r %r\n" % (centre[0], centre[1], centre[2], radius)
    s += "shear_mod 0 %r\nsrho 0 %r\n" % (G, rho)
    return s


def stretched_sphere(n=128, steps=500, mu=0.005, G=1.0, radius=0.3, stretch=1.3, wt_n=1.5, nlayers=5,
                     frames=100000, T=None):
    """Periodic box at rest with a sphere pre-stretched by `stretch` along x:
    xi = c + diag(1/stretch, sqrt(stretch), sqrt(stretch)) (x - c)."""
    if T is None:
        T = frames
    s = _HEAD.format(frames=frames, steps=steps, n=n, T=T, mu=mu)
    s += "wt_n %g\nnlayers %d\nev_trans_mult 0\nn_obj 1\nobject_list 0 1\n" % (wt_n, nlayers)
    s += "basic_specs 0 0.5 0.5 0.5 %r\n" % radius
    s += "extra_specs 0 0 %r 0 0 0 0 0 0 0 0\n" % math.sqrt(stretch)
    s += "shear_mod 0 %r\nsrho 0 1\n" % G
    return s


def multi_sphere(n=24, steps=100, spheres=(), mu=0.01, lid=1.0, wt_n=1.5, nlayers=5, frames=100000, T=None):
    """Lid-driven cavity holding several neo-Hookean spheres (identity maps);
    spheres = [((cx, cy, cz), R, G, rho), ...]."""
    s = cavity(n, steps, mu, lid, frames, T)
    s += "wt_n %g\nnlayers %d\nn_obj %d\n" % (wt_n, nlayers, len(spheres))
    for i, (c, r, G, rho) in enumerate(spheres):
        s += "object_list %d 0\nbasic_specs %d %r %r %r %r\nshear_mod %d %r\nsrho %d %r\n" % (
            i, i, c[0], c[1], c[2], r, i, G, i, rho)
    return s


def ftest(n=16, steps=4, mu=0.01, frames=100000, T=None):
    """The reference's manufactured-solution fluid test (sim_ftest,
    Sim/sim_manager.cc:139-178) on a periodic unit box: a Taylor-Green-like
    velocity decaying as cos(2 pi t) under the matching body force, with the
    exact solution known at every time (has_exact 1)."""
    if T is None:
        T = frames
    s = _HEAD.format(frames=frames, steps=steps, n=n, T=T, mu=mu).replace("sim_type objects", "sim_type ftest")
    return s + "has_exact 1\n"


def wall_sphere(n=24, steps=4, centre=(0.5, 0.5, 0.17), radius=0.12, wall_dist=0.1, gravity=-5.0, G=1.0,
                rho=1.0, frames=100000, T=None):
    """Lid-driven cavity with a sphere close to the bottom wall under gravity:
    the wall repulsion (sim_objects::solid_acceleration, Sim/sim_manager.cc:
    212-295, active within wall_dist of a wall) and the gravity of the solid
    and of the fluid act from the first step."""
    s = cavity_sphere(n, steps, G=G, rho=rho, radius=radius, centre=centre, frames=frames, T=T)
    return s + "wall_dist %r\ngravity %r\n" % (wall_dist, gravity)


def random_scene(seed, sizes=(32, 48, 64, 96), nobj=(1, 8), steps=100, mu=0.01):
    """One seeded multi-sphere cavity scene: radii U(0.08,0.15), centres
    rejection-sampled without overlap and at least 2 dx apart, G log-uniform in
    [0.1,10], solid density U(0.8,1.2), lid speed U(0.5,1.5)."""
    rng = random.Random(seed)
    n = rng.choice(list(sizes))
    k = rng.randint(nobj[0], nobj[1])
    dx = 1.0 / n
    objs = []
    tries = 0
    while len(objs) < k and tries < 10000:
        tries += 1
        r = rng.uniform(0.08, 0.15)
        c = [rng.uniform(r + 4 * dx, 1 - r - 4 * dx) for _ in range(3)]
        ok = all(math.dist(c, o[0]) >= r + o[1] + 2 * dx + 6 * dx for o in objs)
        if ok:
            objs.append((c, r))
    lid = rng.uniform(0.5, 1.5)
    s = "# seed %d\n" % seed + cavity(n, steps, mu, lid)
    s += "wt_n 1.5\nnlayers 5\nn_obj %d\n" % len(objs)
    for i, (c, r) in enumerate(objs):
        G = 10 ** rng.uniform(-1, 1)
        rho = rng.uniform(0.8, 1.2)
        s += "object_list %d 0\nbasic_specs %d %r %r %r %r\nshear_mod %d %r\nsrho %d %r\n" % (
            i, i, c[0], c[1], c[2], r, i, G, i, rho)
    return n, s


def write(path, text):
    with open(path, "w") as f:
        f.write(text)
    return path
