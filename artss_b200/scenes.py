"""XML scene writers in the ARTSS input format (ARTSS src/utility/settings/Settings.cpp).

Every scene the benchmarks and tests use is produced here, as an ordinary ARTSS
XML file that both this package and the reference binary read.  Parameters not
fixed by the workload descriptions (Gauss time constant tau, heat capacity cp,
turbulent Prandtl number, noise step) follow the reference's own Steckler test
XML (tests/navierStokesTempTurb/steckler/Test_NavierStokesTempTurb_Steckler.xml).
"""
from __future__ import annotations

import math
import os
import random
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple


def _f(x: float) -> str:
    return repr(float(x))


@dataclass
class Box:
    """Axis-aligned obstacle in physical coordinates (ox1..oz2)."""
    x1: float
    x2: float
    y1: float
    y2: float
    z1: float
    z2: float
    name: str = "box"


@dataclass
class Scene:
    """One NSTempTurb / Pressure scene.  Field names follow ARTSS XML keys."""
    solver: str = "NSTempTurbSolver"
    nx: int = 64
    ny: int = 64
    nz: int = 64
    X: Tuple[float, float] = (0.0, 2.4)
    Y: Tuple[float, float] = (0.0, 2.4)
    Z: Tuple[float, float] = (0.0, 2.4)
    dt: float = 0.005
    steps: int = 200
    nu: float = 3.1e-5
    kappa: float = 4.2e-5
    beta: float = 3.34e-3
    g: float = -9.81
    diffusion: str = "ColoredGaussSeidel"
    diff_max_iter: int = 100
    diff_tol: float = 1e-7
    cs: float = 0.2
    turbulence: str = "ConstSmagorinsky"  # or "DynamicSmagorinsky" (no parameters)
    # NSTempTurbSolver / NSTempSolver scenes written as NSTempTurbConSolver /
    # NSTempConSolver with a concentration set up exactly like the temperature
    # (gamma = kappa, Sc_T = Pr_T, the same Gauss source, the T boundary
    # conditions for rho)
    concentration: bool = False
    buoyancy_dir: str = "z"
    t_ambient: float = 299.15
    n_level: int = 4
    n_cycle: int = 2
    max_cycle: int = 100
    mg_tol: float = 1e-8
    n_relax: int = 2
    smoother: str = "Jacobi"
    smoother_max_iter: int = 100
    smoother_tol: float = 1e-8
    smoother_w: float = 0.6666666667
    hrr: float = 25.0
    cp: float = 1.0
    source_pos: Tuple[float, float, float] = (1.2, 1.2, 0.3)
    sigma: Tuple[float, float, float] = (0.1, 0.1, 0.1)
    tau: float = 5.0
    pr_t: float = 0.5
    T0: float = 299.15
    noise: bool = True
    noise_range: float = 0.01
    noise_step: float = 0.001
    seed: int = 0
    boundaries: List[Tuple[str, str, str, float]] = field(default_factory=list)
    obstacles: List[Box] = field(default_factory=list)
    obstacle_bcs: List[Tuple[str, str, str, float]] = field(default_factory=list)
    ic: str = "Uniform"
    pressure: str = "VCycleMG"  # or "VCycleMGMixed" (mixed-precision solve to mg_tol, relative)
    ic_params: dict = field(default_factory=dict)  # parameters of ExpSinusProd / GaussBubble / Hat / ...
    force: str = "Buoyancy"  # momentum source force_fct: Buoyancy, Uniform or Zero
    force_value: Tuple[float, float, float] = (0.0, 0.0, 0.0)  # Uniform: val_x, val_y, val_z
    dissipation: bool = False  # temperature source: viscous dissipation (ISource::dissipate)
    # computational domain inside the physical one (X, Y, Z): ((x1, x2), (y1, y2), (z1, z2));
    # nx, ny, nz then count the computational domain's cells
    cd: Optional[Tuple[Tuple[float, float], Tuple[float, float], Tuple[float, float]]] = None
    use_init_values: bool = False  # Buoyancy: use_init_values="Yes" (no ambient temperature value)
    ic_attrs: dict = field(default_factory=dict)  # attributes of <initial_conditions> (LayersT: dir)
    # <adaption dynamic="Yes"> with a Layers class of these parameters (buffer,
    # check_value, timestep, expansion_size); both ARTSS and this library reject it
    adaption: Optional[dict] = None

    @property
    def t_end(self) -> float:
        return self.steps * self.dt

    def inner_cells(self) -> int:
        return self.nx * self.ny * self.nz


def closed_box_bcs(T_type: str = "neumann", T_value: float = 0.0):
    return [
        ("u,v,w", "front,back,bottom,top,left,right", "dirichlet", 0.0),
        ("p", "front,back,bottom,top,left,right", "neumann", 0.0),
        ("T", "front,back,bottom,top,left,right", T_type, T_value),
    ]


def solid_obstacle_bcs():
    return [
        ("u,v,w", "front,back,left,right,top,bottom", "dirichlet", 0.0),
        ("p,T", "front,back,left,right,top,bottom", "neumann", 0.0),
    ]


def plume_box(n: int = 64, steps: int = 200, n_level: int = 4, **kw) -> Scene:
    """Closed 2.4 m box, uniform n^3 grid, 25 kW Gaussian source at (1.2,1.2,0.3):
    the plain FP64 NSTempTurb workload on a 64^3 grid (n=64, 200 steps)."""
    s = Scene(nx=n, ny=n, nz=n, steps=steps, n_level=n_level, boundaries=closed_box_bcs(), **kw)
    return s


def channel_with_cube(nx: int = 256, ny: int = 128, nz: int = 128, steps: int = 500,
                      n_level: int = 4, **kw) -> Scene:
    """6.4 x 3.2 x 3.2 m channel, one 0.4 m cube with its lower corner at
    (1.6, 1.6, 0.2) m, Dirichlet inflow u = 0.5 m/s at x = 0, Neumann outflow at
    x = 6.4 m, 100 kW Gaussian source 0.4 m behind the cube, T0 = 293.15 K."""
    bcs = [
        ("u", "left", "dirichlet", 0.5),
        ("v,w", "left", "dirichlet", 0.0),
        ("u,v,w", "right", "neumann", 0.0),
        ("u,v,w", "front,back,bottom,top", "dirichlet", 0.0),
        ("p", "left,front,back,bottom,top", "neumann", 0.0),
        ("p", "right", "dirichlet", 0.0),
        ("T", "left", "dirichlet", 293.15),
        ("T", "right,front,back,bottom,top", "neumann", 0.0),
    ]
    cube = Box(1.6, 2.0, 1.6, 2.0, 0.2, 0.6, name="cube")
    base = dict(nx=nx, ny=ny, nz=nz, X=(0.0, 6.4), Y=(0.0, 3.2), Z=(0.0, 3.2), dt=0.002,
                steps=steps, n_level=n_level, hrr=100.0, source_pos=(2.4, 1.8, 0.4),
                sigma=(0.2, 0.2, 0.2), T0=293.15, t_ambient=293.15, boundaries=bcs,
                obstacles=[cube], obstacle_bcs=solid_obstacle_bcs())
    base.update(kw)
    return Scene(**base)


def room_with_door(n: int = 32, steps: int = 10, n_level: int = 2, diffusion: str = "Jacobi", **kw) -> Scene:
    """A closed room built from seven touching wall obstacles with a door in
    one wall, heated at the floor centre: the obstacle layout of the
    reference's Steckler test (touching walls exercise the neighbouring-obstacle
    handling of src/domain/Obstacle.cpp:513-859), on a 3.2 m cube of n^3 cells."""
    h = 3.2 / n
    c = lambda k: round(k * h, 12)  # noqa: E731  cell-aligned coordinate
    q = n // 16  # wall thickness in cells
    lo, hi = n // 8, n - n // 8
    x0 = -1.6
    X = lambda k: round(x0 + k * h, 12)  # noqa: E731
    top = (5 * n) // 8
    door_lo, door_hi = (3 * n) // 8, (5 * n) // 8
    door_top = n // 2
    walls = [
        Box(X(lo), X(lo + q), c(0), c(top), X(lo + q), X(hi - q), "left wall"),
        Box(X(lo), X(hi), c(top), c(top + q), X(lo), X(hi), "ceiling"),
        Box(X(lo), X(hi), c(0), c(top), X(hi - q), X(hi), "back wall"),
        Box(X(lo), X(hi), c(0), c(top), X(lo), X(lo + q), "front wall"),
        Box(X(hi - q), X(hi), c(0), c(top), X(lo + q), X(door_lo), "right wall left from door"),
        Box(X(hi - q), X(hi), c(door_top), c(top), X(door_lo), X(door_hi), "right wall above door"),
        Box(X(hi - q), X(hi), c(0), c(top), X(door_hi), X(hi - q), "right wall right from door"),
    ]
    bcs = [
        ("u,v,w", "front,back,bottom,top,left,right", "dirichlet", 0.0),
        ("p", "front,back,bottom,top,left,right", "neumann", 0.0),
        ("T", "front,back,top,left,right", "dirichlet", 299.14),
        ("T", "bottom", "neumann", 0.0),
    ]
    base = dict(nx=n, ny=n, nz=n, X=(-1.6, 1.6), Y=(0.0, 3.2), Z=(-1.6, 1.6), dt=0.01, steps=steps,
                n_level=n_level, diffusion=diffusion, buoyancy_dir="y", hrr=50.3, source_pos=(0.0, 0.2, 0.0),
                sigma=(0.25, 0.6, 0.25), T0=299.14, t_ambient=299.14, boundaries=bcs, obstacles=walls,
                obstacle_bcs=solid_obstacle_bcs(), n_relax=4, mg_tol=1e-7, smoother_tol=1e-7, noise_step=0.1,
                noise_range=1.0)
    base.update(kw)
    return Scene(**base)


def random_boxes(n_cells: Tuple[int, int, int], lo: int, hi: int, count: int, seed: int,
                 spacing: Tuple[float, float, float], origin=(0.0, 0.0, 0.0),
                 levels: int = 0, max_tries: int = 10000) -> List[Box]:
    """Axis-aligned boxes with edges uniform in [lo, hi] cells at uniform
    positions, rejected when they touch or overlap (with a one-cell gap at every
    multigrid level), since the reference's list construction is only well
    defined for obstacles that stay apart after restriction
    (src/domain/Multigrid.cpp:495-512 keeps duplicates)."""
    rng = random.Random(seed)
    boxes_idx: List[Tuple[int, int, int, int, int, int]] = []
    gap = 2 ** (levels + 1)
    tries = 0
    while len(boxes_idx) < count and tries < max_tries:
        tries += 1
        e = [rng.randint(lo, hi) for _ in range(3)]
        if any(e[a] > n_cells[a] - 2 * gap for a in range(3)):
            continue
        s = [rng.randint(gap, n_cells[a] - e[a] - gap) for a in range(3)]
        # snap to multiples of 2^levels so coarse boxes keep their shape
        q = 2 ** levels
        s = [(s[a] // q) * q for a in range(3)]
        e = [max(q, (e[a] // q) * q) for a in range(3)]
        cand = (s[0], s[0] + e[0], s[1], s[1] + e[1], s[2], s[2] + e[2])
        ok = True
        for b in boxes_idx:
            if all(cand[2 * a] < b[2 * a + 1] + gap and b[2 * a] < cand[2 * a + 1] + gap for a in range(3)):
                ok = False
                break
        if ok:
            boxes_idx.append(cand)
    out = []
    for n, b in enumerate(boxes_idx):
        out.append(Box(origin[0] + b[0] * spacing[0], origin[0] + b[1] * spacing[0],
                       origin[1] + b[2] * spacing[1], origin[1] + b[3] * spacing[1],
                       origin[2] + b[4] * spacing[2], origin[2] + b[5] * spacing[2], name=f"box{n}"))
    return out


def poisson_boxes(n: int = 256, seed: int = 0, n_level: int = 5, **kw) -> Scene:
    """Pure-Neumann pressure problem on a unit-spacing n^3 grid with 1-6
    axis-aligned box obstacles whose edges are uniform in [8, 48] cells at
    uniform positions (count, sizes and positions from `seed`): the
    mixed-precision pressure workload at n = 256.  The right-hand side is not
    part of the scene; poisson_rhs() draws it."""
    rng = random.Random(10007 * seed + 17)
    count = rng.randint(1, 6)
    lo, hi = max(2, 8 * n // 256), max(3, 48 * n // 256)
    boxes = random_boxes((n, n, n), lo, hi, count, seed, (1.0, 1.0, 1.0), levels=n_level - 1)
    bcs = [("p", "front,back,bottom,top,left,right", "neumann", 0.0)]
    obcs = [("p", "front,back,left,right,top,bottom", "neumann", 0.0)]
    base = dict(solver="PressureSolver", nx=n, ny=n, nz=n, X=(0.0, float(n)), Y=(0.0, float(n)), Z=(0.0, float(n)),
                dt=1.0, steps=1, n_level=n_level, boundaries=bcs, obstacles=boxes, obstacle_bcs=obcs, noise=False,
                ic="Zero")
    base.update(kw)
    return Scene(**base)


def poisson_rhs(inner, size: int, seed: int):
    """Seeded N(0, 1) right-hand side on the inner cells, projected to zero
    mean over them (every other cell 0)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    b = np.zeros(size)
    v = rng.standard_normal(len(inner))
    b[inner] = v - v.mean()
    return b


VELOCITY_SOLVERS = ("AdvectionSolver", "AdvectionDiffusionSolver", "DiffusionSolver", "DiffusionTurbSolver")


def velocity_scene(solver: str, n: int = 32, steps: int = 5, diffusion: str = "Jacobi", **kw) -> Scene:
    """A velocity-only scene of the reference's test family (tests/diffusion,
    tests/advection, tests/diffusionTurb): a 2 x 2 x 1 m box with Dirichlet
    u = v = w = 0 walls, n x n x n/2 cells, initial u, v, w from ExpSinusProd
    (diffusion solvers) or GaussBubble (advection solvers)."""
    if solver not in VELOCITY_SOLVERS:
        raise ValueError(solver)
    if solver in ("AdvectionSolver", "AdvectionDiffusionSolver"):
        ic, params = "GaussBubble", {"u_lin": 0.5, "v_lin": 0.5, "w_lin": 0.25, "x_shift": 0.6, "y_shift": 0.7,
                                     "z_shift": 0.5, "l": 0.25}
    else:
        ic, params = "ExpSinusProd", {"l": 2.5}
    base = dict(solver=solver, nx=n, ny=n, nz=max(n // 2, 2), X=(0.0, 2.0), Y=(0.0, 2.0), Z=(0.0, 1.0), dt=0.0125,
                steps=steps, nu=0.001, diffusion=diffusion, diff_tol=1e-7, diff_max_iter=100,
                boundaries=[("u,v,w", "front,back,left,right,bottom,top", "dirichlet", 0.0)], noise=False, ic=ic,
                ic_params=params)
    base.update(kw)
    return Scene(**base)


def pressure_scene(n: int = 32, n_level: int = 4, steps: int = 2, **kw) -> Scene:
    """PressureSolver scene of the reference's tests/pressure family: a 2 m cube,
    n^3 cells, Dirichlet p = 0 on every wall, rhs = sin(l pi x) sin(l pi y)
    sin(l pi z) with l = 2 (SinSinSin), VCycleMG V(4,4) to 1e-7."""
    base = dict(solver="PressureSolver", nx=n, ny=n, nz=n, X=(0.0, 2.0), Y=(0.0, 2.0), Z=(0.0, 2.0), dt=0.1,
                steps=steps, n_level=n_level, max_cycle=100, mg_tol=1e-7, n_relax=4, smoother_max_iter=100,
                smoother_tol=1e-7, boundaries=[("p", "front,back,left,right,bottom,top", "dirichlet", 0.0)],
                noise=False, ic="SinSinSin", ic_params={"l": 2.0})
    base.update(kw)
    return Scene(**base)


def layered_channel(nx: int = 64, ny: int = 16, nz: int = 32, steps: int = 4, n_level: int = 4,
                    use_init_values: bool = False, **kw) -> Scene:
    """A computational domain inside a longer physical one: the channel runs
    0..48 m in x, the solver works on x in 16..24 m (nx cells, so the physical
    domain holds 6 nx cells plus ghosts); y in -2..2 m, z in -3..3 m.  The
    temperature starts in four horizontal layers (LayersT across y), a Gauss
    source near the floor heats it, buoyancy acts along y.  No-slip floor,
    ceiling and side walls, open ends (Neumann velocity, p = 0)."""
    base = dict(solver="NSTempTurbSolver", nx=nx, ny=ny, nz=nz, X=(0.0, 48.0), Y=(-2.0, 2.0), Z=(-3.0, 3.0),
                cd=((16.0, 24.0), (-2.0, 2.0), (-3.0, 3.0)), dt=0.05, steps=steps, nu=2.5e-5, kappa=3.3e-5,
                beta=3.28e-3, diffusion="Jacobi", diff_tol=1e-7, n_level=n_level, n_cycle=2, max_cycle=100,
                mg_tol=1e-7, n_relax=4, smoother="Jacobi", smoother_tol=1e-7, buoyancy_dir="y",
                use_init_values=use_init_values, t_ambient=300.0, hrr=5000.0, cp=1.0,
                source_pos=(20.0, -2.0, 0.0), sigma=(0.75, 1.0, 0.75), tau=5.0, noise=False, ic="LayersT",
                ic_attrs={"dir": "y"},
                ic_params={"n_layers": 4, "border_1": -1.0, "border_2": 0.0, "border_3": 1.0,
                           "value_1": 300.5, "value_2": 301.0, "value_3": 302.5, "value_4": 304.0},
                boundaries=[("u,v,w", "front,back,bottom,top", "dirichlet", 0.0),
                            ("u,v,w", "left,right", "neumann", 0.0),
                            ("p", "front,back,bottom,top", "neumann", 0.0),
                            ("p", "left,right", "dirichlet", 0.0),
                            ("T", "front,back,bottom,top,left,right", "neumann", 0.0)])
    base.update(kw)
    return Scene(**base)


def inset_box(n: int = 32, steps: int = 4, n_level: int = 3, **kw) -> Scene:
    """A computational domain strictly inside the physical domain on every
    axis (x 4..8 of 0..12, y 1..5 of 0..6, z 2..4 of 0..6 m; n x n x n/2 cells
    of 4/n m) with a solid block inside it, colored Gauss-Seidel diffusion and
    the plume source: every boundary condition acts on faces interior to the
    physical arrays."""
    h = 4.0 / n
    block = Box(5.5, 5.5 + 8 * h, 1.0, 1.0 + 6 * h, 2.5, 2.5 + 4 * h, "block")
    base = dict(nx=n, ny=n, nz=n // 2, X=(0.0, 12.0), Y=(0.0, 6.0), Z=(0.0, 6.0),
                cd=((4.0, 8.0), (1.0, 5.0), (2.0, 4.0)), steps=steps, n_level=n_level, dt=0.01,
                source_pos=(6.0, 2.0, 3.0), sigma=(0.4, 0.4, 0.4), hrr=50.0, buoyancy_dir="y",
                boundaries=closed_box_bcs(), obstacles=[block], obstacle_bcs=solid_obstacle_bcs())
    base.update(kw)
    return Scene(**base)


def burgers_scene(n: int = 32, nz: int = 1, steps: int = 4, **kw) -> Scene:
    """AdvectionDiffusionSolver on the ExpSinusSum state (the reference's Burgers
    test family, tests/burgers): a periodic 2 pi box, n x n x nz cells; nz = 1
    is the 2-D form (u = -v = sin(x + y), w = 0), larger nz the 3-D one
    (u = sin(x + y + z), v = w = -u / 2)."""
    L = 2.0 * math.pi
    base = dict(solver="AdvectionDiffusionSolver", nx=n, ny=n, nz=nz, X=(0.0, L), Y=(0.0, L),
                Z=(0.0, L if nz > 1 else L / n), dt=0.01, steps=steps, nu=0.05, diffusion="Jacobi", diff_tol=1e-7,
                diff_max_iter=100, noise=False, ic="ExpSinusSum",
                boundaries=[("u,v,w", "front,back,left,right,bottom,top", "periodic", 0.0)])
    base.update(kw)
    return Scene(**base)


NS_SOLVERS = ("NSSolver", "NSTurbSolver")


def ns_scene(kind: str, solver: str = "NSSolver", n: int = 32, steps: int = 4, **kw) -> Scene:
    """Isothermal Navier-Stokes scenes of the reference's test family
    (tests/navierStokes, tests/navierStokesTurb), in 3-D:
      cavity   lid-driven unit cube, u = 1 on the top wall, n x n x n/2 cells;
      mcdermott  periodic 2 pi box with the McDermott vortex array (A = 2);
      vortex   periodic box centred on the origin with one travelling vortex;
      channel  Drift start u = 0.5 between no-slip walls, periodic in x,
               with a uniform x force (which NSSolver never sets, as in the
               reference, whose force_source runs only for the temperature solvers)."""
    if solver not in NS_SOLVERS:
        raise ValueError(solver)
    nz = max(n // 2, 2)
    periodic = [("u,v,w", "front,back,left,right,bottom,top", "periodic", 0.0),
                ("p", "front,back,left,right,bottom,top", "periodic", 0.0)]
    base = dict(solver=solver, nx=n, ny=n, nz=nz, steps=steps, noise=False, diffusion="Jacobi", diff_tol=1e-7,
                force="Zero", buoyancy_dir="x,y,z", n_level=3, smoother_tol=1e-7)
    if kind == "cavity":
        base.update(X=(0.0, 1.0), Y=(0.0, 1.0), Z=(0.0, 0.5), dt=0.005, nu=0.01, ic="Zero",
                    boundaries=[("u", "top", "dirichlet", 1.0), ("u", "front,back,left,right,bottom", "dirichlet", 0.0),
                                ("v,w", "front,back,left,right,bottom,top", "dirichlet", 0.0),
                                ("p", "top", "dirichlet", 0.0), ("p", "front,back,left,right,bottom", "neumann", 0.0)])
    elif kind == "mcdermott":
        L = 2.0 * math.pi
        base.update(X=(0.0, L), Y=(0.0, L), Z=(0.0, L / 2), dt=0.01, nu=0.1, ic="McDermott", ic_params={"A": 2.0},
                    boundaries=periodic)
    elif kind == "vortex":
        base.update(X=(-0.16, 0.16), Y=(-0.16, 0.16), Z=(-0.08, 0.08), dt=0.002, nu=1e-4, ic="Vortex",
                    ic_params={"u_lin": 0.5, "v_lin": 0.0, "w_lin": 0.1, "pa": 0.0, "rhoa": 1.0},
                    boundaries=periodic)
    elif kind == "channel":
        base.update(X=(0.0, 2.0), Y=(0.0, 1.0), Z=(0.0, 1.0), dt=0.01, nu=0.01, ic="Drift",
                    ic_params={"u_lin": 0.5, "v_lin": 0.0, "w_lin": 0.0, "pa": 0.0}, force="Uniform",
                    buoyancy_dir="x", force_value=(0.2, 0.0, 0.0),
                    boundaries=[("u,v,w", "left,right", "periodic", 0.0),
                                ("u,v,w", "front,back,bottom,top", "dirichlet", 0.0),
                                ("p", "left,right", "periodic", 0.0), ("p", "front,back,bottom,top", "neumann", 0.0)])
    else:
        raise ValueError(kind)
    base.update(kw)
    return Scene(**base)


def plume_ensemble(count: int = 64, seed: int = 0, steps: int = 100, sizes=(32, 48, 64, 96, 128)) -> List[Scene]:
    """The ensemble workload: `count` closed plume boxes whose cell counts per
    axis are drawn from `sizes`, 0.0375 m cells, heat release U[10, 150] kW
    centred at U[0.2, 0.8] of the extent (0.3 of the height), 0-3 box
    obstacles, dt 0.005 s, the mixed-precision pressure solve to 1e-8
    relative or 20 cycles per step."""
    rng = random.Random(seed)
    out = []
    h = 0.0375
    for n in range(count):
        nx, ny, nz = (rng.choice(sizes) for _ in range(3))
        ext = (nx * h, ny * h, nz * h)
        sc = Scene(nx=nx, ny=ny, nz=nz, X=(0.0, ext[0]), Y=(0.0, ext[1]), Z=(0.0, ext[2]), dt=0.005, steps=steps,
                   n_level=4, boundaries=closed_box_bcs(), hrr=rng.uniform(10.0, 150.0),
                   source_pos=(rng.uniform(0.2, 0.8) * ext[0], rng.uniform(0.2, 0.8) * ext[1], 0.3 * ext[2]),
                   seed=rng.randint(0, 10 ** 6), pressure="VCycleMGMixed", max_cycle=20)
        sc.obstacles = random_boxes((nx, ny, nz), 8, 16, rng.randint(0, 3), rng.randint(0, 10 ** 6), (h, h, h),
                                    levels=3)
        sc.obstacle_bcs = solid_obstacle_bcs()
        out.append(sc)
    return out


def to_xml(s: Scene) -> str:
    L = []
    a = L.append
    a('<?xml version="1.0" encoding="UTF-8" ?>')
    a("<ARTSS>")
    a("  <physical_parameters>")
    a(f"    <t_end> {_f(s.t_end)} </t_end>")
    a(f"    <dt> {_f(s.dt)} </dt>")
    velocity_only = s.solver in VELOCITY_SOLVERS
    # NSTempSolver and NSSolver (src/solver/NSTempSolver.cpp, NSSolver.cpp) read
    # no turbulence blocks; NSSolver and NSTurbSolver carry no temperature
    turbulent = s.solver not in ("NSTempSolver", "NSSolver")
    temperature = s.solver not in NS_SOLVERS + ("PressureSolver",)
    if velocity_only:
        if s.solver != "AdvectionSolver":
            a(f"    <nu> {_f(s.nu)} </nu>")
    elif s.solver != "PressureSolver":
        a(f"    <nu> {_f(s.nu)} </nu>")
        a(f"    <beta> {_f(s.beta)} </beta>")
        a(f"    <g> {_f(s.g)} </g>")
        a("    <rhoa> 1 </rhoa>")
        if temperature:
            a(f"    <kappa> {_f(s.kappa)} </kappa>")
        if s.concentration:
            a(f"    <gamma> {_f(s.kappa)} </gamma>")
    a("  </physical_parameters>")
    description = s.solver
    if s.concentration:
        if s.solver not in ("NSTempTurbSolver", "NSTempSolver"):
            raise ValueError("concentration needs NSTempTurbSolver or NSTempSolver")
        description = "NSTempTurbConSolver" if s.solver == "NSTempTurbSolver" else "NSTempConSolver"
    a(f'  <solver description="{description}" >')

    def turbulence_block():
        if s.turbulence == "DynamicSmagorinsky":
            a('    <turbulence type="DynamicSmagorinsky">')
        else:
            a('    <turbulence type="ConstSmagorinsky">')
            a(f"      <Cs> {_f(s.cs)} </Cs>")
        a("    </turbulence>")

    def diffusion_block(tag_field: str, indent: str, typ: str, max_iter: int, tol: float, w: float):
        a(f'{indent}<diffusion type="{typ}" field="{tag_field}">')
        a(f"{indent}  <max_iter> {max_iter} </max_iter>")
        a(f"{indent}  <tol_res> {_f(tol)} </tol_res>")
        a(f"{indent}  <w> {_f(w)} </w>")
        a(f"{indent}</diffusion>")

    if velocity_only:
        if s.solver in ("AdvectionSolver", "AdvectionDiffusionSolver"):
            a('    <advection type="SemiLagrangian" field="u,v,w">')
            a("    </advection>")
        if s.solver != "AdvectionSolver":
            diffusion_block("u,v,w", "    ", s.diffusion, s.diff_max_iter, s.diff_tol, 1.0)
        if s.solver == "DiffusionTurbSolver":
            turbulence_block()
    elif s.solver != "PressureSolver":
        a('    <advection type="SemiLagrangian" field="u,v,w">')
        a("    </advection>")
        diffusion_block("u,v,w", "    ", s.diffusion, s.diff_max_iter, s.diff_tol, 1.0)
        if turbulent:
            turbulence_block()
        if s.force == "Buoyancy":
            a(f'    <source type="ExplicitEuler" force_fct="Buoyancy" dir="{s.buoyancy_dir}" '
              f'use_init_values="{"Yes" if s.use_init_values else "No"}">')
            if not s.use_init_values:
                a(f"      <ambient_temperature_value> {_f(s.t_ambient)} </ambient_temperature_value>")
        elif s.force == "Uniform":
            a(f'    <source type="ExplicitEuler" force_fct="Uniform" dir="{s.buoyancy_dir}">')
            for ax, val in zip("xyz", s.force_value):
                a(f"      <val_{ax}> {_f(val)} </val_{ax}>")
        else:
            a(f'    <source type="ExplicitEuler" force_fct="{s.force}" dir="{s.buoyancy_dir}">')
        a("    </source>")
    if not velocity_only:
        a(f'    <pressure type="{s.pressure}" field="p">')
        a(f"      <n_level> {s.n_level} </n_level>")
        a(f"      <n_cycle> {s.n_cycle} </n_cycle>")
        a(f"      <max_cycle> {s.max_cycle} </max_cycle>")
        a(f"      <tol_res> {_f(s.mg_tol)} </tol_res>")
        a(f"      <n_relax> {s.n_relax} </n_relax>")
        diffusion_block("p", "      ", s.smoother, s.smoother_max_iter, s.smoother_tol, s.smoother_w)
        a("    </pressure>")
    if temperature and not velocity_only:
        a("    <temperature>")
        a('      <advection type="SemiLagrangian" field="T">')
        a("      </advection>")
        diffusion_block("T", "      ", s.diffusion, s.diff_max_iter, s.diff_tol, 1.0)
        if turbulent:
            a('      <turbulence include="Yes">')
            a(f"        <Pr_T> {_f(s.pr_t)} </Pr_T>")
            a("      </turbulence>")
        a(f'      <source type="ExplicitEuler" dir="{s.buoyancy_dir}" temp_fct="Gauss" '
          f'dissipation="{"Yes" if s.dissipation else "No"}" random="No">')
        a(f"        <HRR> {_f(s.hrr)} </HRR>")
        a(f"        <cp> {_f(s.cp)} </cp>")
        a(f"        <x0> {_f(s.source_pos[0])} </x0>")
        a(f"        <y0> {_f(s.source_pos[1])} </y0>")
        a(f"        <z0> {_f(s.source_pos[2])} </z0>")
        a(f"        <sigma_x> {_f(s.sigma[0])} </sigma_x>")
        a(f"        <sigma_y> {_f(s.sigma[1])} </sigma_y>")
        a(f"        <sigma_z> {_f(s.sigma[2])} </sigma_z>")
        a(f"        <tau> {_f(s.tau)} </tau>")
        a("      </source>")
        a("    </temperature>")
        if s.concentration:
            a("    <concentration>")
            a('      <advection type="SemiLagrangian" field="rho">')
            a("      </advection>")
            diffusion_block("rho", "      ", s.diffusion, s.diff_max_iter, s.diff_tol, 1.0)
            if turbulent:
                a('      <turbulence include="Yes">')
                a(f"        <Sc_T> {_f(s.pr_t)} </Sc_T>")
                a("      </turbulence>")
            a(f'      <source type="ExplicitEuler" dir="{s.buoyancy_dir}" con_fct="Gauss" random="No">')
            a(f"        <HRR> {_f(s.hrr)} </HRR>")
            a(f"        <cp> {_f(s.cp)} </cp>")
            a(f"        <x0> {_f(s.source_pos[0])} </x0>")
            a(f"        <y0> {_f(s.source_pos[1])} </y0>")
            a(f"        <z0> {_f(s.source_pos[2])} </z0>")
            a(f"        <sigma_x> {_f(s.sigma[0])} </sigma_x>")
            a(f"        <sigma_y> {_f(s.sigma[1])} </sigma_y>")
            a(f"        <sigma_z> {_f(s.sigma[2])} </sigma_z>")
            a(f"        <tau> {_f(s.tau)} </tau>")
            a("      </source>")
            a("    </concentration>")
    a('    <solution available="No">')
    a("    </solution>")
    a("  </solver>")
    a(f'  <domain_parameters enable_computational_domain="{"Yes" if s.cd else "No"}">')
    for ax, (lo, hi) in zip("XYZ", (s.X, s.Y, s.Z)):
        a(f"    <{ax}1> {_f(lo)} </{ax}1>")
        a(f"    <{ax}2> {_f(hi)} </{ax}2>")
    if s.cd:
        for ax, (lo, hi) in zip("xyz", s.cd):
            a(f"    <{ax}1> {_f(lo)} </{ax}1>")
            a(f"    <{ax}2> {_f(hi)} </{ax}2>")
    a(f"    <nx> {s.nx} </nx>")
    a(f"    <ny> {s.ny} </ny>")
    a(f"    <nz> {s.nz} </nz>")
    a("  </domain_parameters>")
    if s.adaption:
        a('  <adaption dynamic="Yes" data_extraction="No">')
        a('    <class name="Layers">')
        for k, v in s.adaption.items():
            a(f"      <{k}> {_f(v)} </{k}>")
        a("    </class>")
        a("  </adaption>")
    else:
        a('  <adaption dynamic="No" data_extraction="No"> </adaption>')
    a('  <data_assimilation enabled="No" />')
    def with_rho(bcs):
        out = list(bcs)
        if s.concentration:
            out += [("rho", patch, typ, val) for fld, patch, typ, val in bcs if "T" in fld.split(",")]
        return out

    a("  <boundaries>")
    for fld, patch, typ, val in with_rho(s.boundaries):
        a(f'    <boundary field="{fld}" patch="{patch}" type="{typ}" value="{_f(val)}" />')
    a("  </boundaries>")
    if s.obstacles:
        a('  <obstacles enabled="Yes">')
        for b in s.obstacles:
            a(f'    <obstacle name="{b.name}">')
            a(f'      <geometry ox1="{_f(b.x1)}" ox2="{_f(b.x2)}" oy1="{_f(b.y1)}" oy2="{_f(b.y2)}"'
              f' oz1="{_f(b.z1)}" oz2="{_f(b.z2)}"/>')
            for fld, patch, typ, val in with_rho(s.obstacle_bcs or solid_obstacle_bcs()):
                a(f'      <boundary field="{fld}" patch="{patch}" type="{typ}" value="{_f(val)}"/>')
            a("    </obstacle>")
        a("  </obstacles>")
    else:
        a('  <obstacles enabled="No"/>')
    a('  <surfaces enabled="No"/>')
    # Uniform and LayersT take the seeded noise on T (SolverController.cpp:167-180)
    noisy = s.noise and s.ic in ("Uniform", "LayersT")
    attrs = "".join(f' {k}="{v}"' for k, v in s.ic_attrs.items())
    a(f'  <initial_conditions usr_fct="{s.ic}"{attrs} random="{"Yes" if noisy else "No"}">')
    if s.ic == "Uniform":
        a(f"    <val> {_f(s.T0)} </val>")
    for k, v in s.ic_params.items():
        a(f"    <{k}> {_f(v)} </{k}>")
    if noisy:
        a('    <random absolute="Yes" custom_seed="Yes" custom_steps="Yes">')
        a(f"      <seed> {s.seed} </seed>")
        a(f"      <step_size> {_f(s.noise_step)} </step_size>")
        a(f"      <range> {_f(s.noise_range)} </range>")
        a("    </random>")
    a("  </initial_conditions>")
    a('  <visualisation save_vtk="No" save_csv="No">')
    a("  </visualisation>")
    a('  <logging file="artss.log" level="info">')
    a("  </logging>")
    a("</ARTSS>")
    return "\n".join(L) + "\n"


def write(s: Scene, path: str) -> str:
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        f.write(to_xml(s))
    return path
