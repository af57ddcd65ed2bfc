"""Synthetic scenario builders with the shapes of the benchmark workloads.

Every builder returns a `LeapFrogTimeIntegrator` assembled from the
reference-API mirror plus a dict of metadata (dt inputs, counts).  Geometry
follows the reference's example scripts: lattice fluid at (i+½)dx, boundary
walls as 3-layer `DynamicBoundarySystem`s (DambreakWall.jl:107-172 pattern),
the elasto-plastic column with a dynamic bottom and a ghost-mirrored left
wall (EP_ColumnCollapse.jl:13-129).  Inputs the reference scripts do not
build themselves are constructed here:
  * hydrostatic initial density (inverse of the Tait EOS,
    src/StateUpdaters.jl:117) for the dam breaks;
  * geostatic K0 initial stress for the columns (the reference starts EP
    stress at zero, src/Particles.jl:410).
"""
from __future__ import annotations

import math

import numpy as np

from .model import (BasicParticleSystem, CauchyFluidPfn, CubicSplineKernel, DynamicBoundarySystem,
                    ElastoPlasticParticleSystem, ElastoPlasticStressUpdater, FluidParticleSystem, FluidPfn,
                    FluidSolidPfn, HookeLawStressUpdater,
                    GhostCopier, GhostEntry, GhostParticleSystem, HouseholderReflect, LeapFrogTimeIntegrator,
                    LinearEOSUpdater, ProbeParticleSystem, StaticBoundarySystem,
                    RK4TimeIntegrator, StrainRatePfn, InterpolateFieldFn, VirtualNormUpdater,
                    VirtualParticleSystem, PrescribedVelocityUpdater, StrainRateVorticityPfn, StressParticleSystem, SystemInteraction,
                    TaitEOSUpdater, ViscoPlasticMCStressUpdater, WenlandC2Kernel, XSPHPfn, ZeroFieldUpdater)

G = 9.81


def _tait_pressure(rho, rho0, c, gamma):
    return rho0 * c * c / gamma * ((rho / rho0) ** gamma - 1.0)


def _wall(name, pts, mass, c, rho0):
    ps = BasicParticleSystem(name, len(pts), pts.shape[1], mass, c)
    ps.x[:] = pts
    ps.rho[:] = rho0
    return ps


# ------------------------------------------------------------ dam break 2-D

def dambreak_2d(nx=50, ny=100, dx=0.02, tank=(4.0, 4.0), layers=3, rho0=1000.0, gamma=7.0,
                alpha=0.01, beta=0.0, hfac=1.2, cfl=0.2, wall_beta=3.0):
    """2-D weakly-compressible dam break (FP64 plain single instance).

    Water column nx×ny at spacing dx in the lower-left corner of a tank of
    `tank` metres with `layers` rows of boundary particles per wall."""
    W, H = tank
    col_h = ny * dx
    c0 = 10.0 * math.sqrt(2.0 * G * col_h)
    h = hfac * dx
    mass = rho0 * dx * dx
    ii, jj = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    x = np.stack([(ii.ravel() + 0.5) * dx, (jj.ravel() + 0.5) * dx], axis=1)
    fluid = FluidParticleSystem("fluid", len(x), 2, mass, c0, source_v=[0.0, -G],
                                state_updater=TaitEOSUpdater(rho0, gamma=gamma))
    fluid.x[:] = x
    fluid.rho[:] = rho0 * (1.0 + gamma * G * (col_h - x[:, 1]) / (c0 * c0)) ** (1.0 / gamma)
    fluid.p[:] = _tait_pressure(fluid.rho, rho0, c0, gamma)

    nwx = int(round(W / dx)) + 6
    nwy = int(round(H / dx))
    lay = np.arange(layers)
    xs = -2.5 * dx + np.arange(nwx) * dx
    ys = (np.arange(nwy) + 0.5) * dx
    floor = np.array([(xv, -(l + 0.5) * dx) for l in lay for xv in xs])
    top = np.array([(xv, H + (l + 0.5) * dx) for l in lay for xv in xs])
    left = np.array([(-(l + 0.5) * dx, yv) for l in lay for yv in ys])
    right = np.array([(W + (l + 0.5) * dx, yv) for l in lay for yv in ys])
    walls = [("floor", floor, (0.0, 1.0), (0.0, 0.0)), ("left", left, (1.0, 0.0), (0.0, 0.0)),
             ("right", right, (-1.0, 0.0), (W, 0.0)), ("top", top, (0.0, -1.0), (0.0, H))]
    kernel = CubicSplineKernel(h, ndims=2)
    pfn = FluidPfn(alpha, beta, h)
    systems = [fluid]
    inters = [SystemInteraction(kernel, pfn, fluid)]
    for name, pts, nrm, pt in walls:
        inner = _wall(name, pts, mass, c0, rho0)
        systems.append(inner)
        inters.append(SystemInteraction(kernel, pfn, fluid, DynamicBoundarySystem(inner, nrm, pt, wall_beta)))
    lf = LeapFrogTimeIntegrator(systems, inters)
    meta = dict(workload="dambreak_2d", n_fluid=fluid.n, n_boundary=sum(s.n for s in systems[1:]),
                h=h, c0=c0, cfl=cfl, dt=cfl * h / c0, ndims=2)
    return lf, meta


# ------------------------------------------------------------ dam break 3-D

def dambreak_3d(nx=100, ny=50, nz=200, dx=0.01, tank=(4.0, 1.0, 4.0), layers=3, rho0=1000.0, gamma=7.0,
                alpha=0.01, beta=0.0, hfac=1.2, cfl=0.2, wall_beta=3.0):
    """3-D dam break: fluid block nx×ny×nz (z vertical, as dambreak_3d.jl)
    in a tank of `tank` metres with 3-layer dynamic walls on all six faces."""
    X, Y, Z = tank
    col_h = nz * dx
    c0 = 10.0 * math.sqrt(2.0 * G * col_h)
    h = hfac * dx
    mass = rho0 * dx ** 3
    ii, jj, kk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    x = np.stack([(ii.ravel() + 0.5) * dx, (jj.ravel() + 0.5) * dx, (kk.ravel() + 0.5) * dx], axis=1)
    fluid = FluidParticleSystem("fluid", len(x), 3, mass, c0, source_v=[0.0, 0.0, -G],
                                state_updater=TaitEOSUpdater(rho0, gamma=gamma))
    fluid.x[:] = x
    fluid.rho[:] = rho0 * (1.0 + gamma * G * (col_h - x[:, 2]) / (c0 * c0)) ** (1.0 / gamma)
    fluid.p[:] = _tait_pressure(fluid.rho, rho0, c0, gamma)

    nX, nY, nZ = (int(round(v / dx)) for v in (X, Y, Z))
    ext_x = -2.5 * dx + np.arange(nX + 6) * dx
    ext_y = -2.5 * dx + np.arange(nY + 6) * dx
    in_y = (np.arange(nY) + 0.5) * dx
    in_z = (np.arange(nZ) + 0.5) * dx
    ext_x_l = ext_x
    layers_off = [(l + 0.5) * dx for l in range(layers)]

    def plane(a, b, fixed_axis, fixed_vals):
        A, B = np.meshgrid(a, b, indexing="ij")
        out = []
        for f in fixed_vals:
            cols = [None, None, None]
            free = [ax for ax in range(3) if ax != fixed_axis]
            cols[free[0]] = A.ravel()
            cols[free[1]] = B.ravel()
            cols[fixed_axis] = np.full(A.size, f)
            out.append(np.stack(cols, axis=1))
        return np.concatenate(out)

    walls = [
        ("floor", plane(ext_x, ext_y, 2, [-o for o in layers_off]), (0, 0, 1.0), (0, 0, 0.0)),
        ("ceiling", plane(ext_x, ext_y, 2, [Z + o for o in layers_off]), (0, 0, -1.0), (0, 0, Z)),
        ("left", plane(in_y, in_z, 0, [-o for o in layers_off]), (1.0, 0, 0), (0.0, 0, 0)),
        ("right", plane(in_y, in_z, 0, [X + o for o in layers_off]), (-1.0, 0, 0), (X, 0, 0)),
        ("front", plane(ext_x_l, in_z, 1, [-o for o in layers_off]), (0, 1.0, 0), (0, 0.0, 0)),
        ("back", plane(ext_x_l, in_z, 1, [Y + o for o in layers_off]), (0, -1.0, 0), (0, Y, 0)),
    ]
    kernel = CubicSplineKernel(h, ndims=3)
    pfn = FluidPfn(alpha, beta, h)
    systems = [fluid]
    inters = [SystemInteraction(kernel, pfn, fluid)]
    for name, pts, nrm, pt in walls:
        inner = _wall(name, pts, mass, c0, rho0)
        systems.append(inner)
        inters.append(SystemInteraction(kernel, pfn, fluid, DynamicBoundarySystem(inner, nrm, pt, wall_beta)))
    lf = LeapFrogTimeIntegrator(systems, inters)
    meta = dict(workload="dambreak_3d", n_fluid=fluid.n, n_boundary=sum(s.n for s in systems[1:]),
                h=h, c0=c0, cfl=cfl, dt=cfl * h / c0, ndims=3)
    return lf, meta


# ------------------------------------- dam breaks with a static (LJ) wall

def dambreak_lj_2d(nfx=50, nfy=50, nbx=150, nby=80, dx=0.5, rho0=1000.0, alpha=0.01, beta=0.0, hfac=1.2,
                   cfl=0.05, column_height=None):
    """2-D dam break in a single-layer Lennard-Jones wall (dambreak.jl
    layout): an nfx×nfy fluid block at ((i+½)dx, (j+½)dx), i outer, at rest
    with ρ = ρ0 and p from the Tait EOS (zero), in a box nbx·dx wide and
    nby·dx tall whose wall particles (bottom and top rows from i = -1 to nbx,
    then the left and right columns) form one BasicParticleSystem wrapped as
    StaticBoundarySystem(boundary, dx).  c0 = 10·sqrt(2 g H) with H the
    column height (25 m in the script)."""
    H = nfy * dx if column_height is None else column_height
    c0 = 10.0 * math.sqrt(2.0 * G * H)
    h = hfac * dx
    mass = rho0 * dx * dx
    ii, jj = np.meshgrid(np.arange(nfx), np.arange(nfy), indexing="ij")
    fluid = FluidParticleSystem("fluid", nfx * nfy, 2, mass, c0, source_v=[0.0, -G],
                                state_updater=TaitEOSUpdater(rho0))
    fluid.x[:, 0] = (ii.ravel() + 0.5) * dx
    fluid.x[:, 1] = (jj.ravel() + 0.5) * dx
    fluid.rho[:] = rho0
    fluid.p[:] = _tait_pressure(fluid.rho, rho0, c0, 7.0)
    W, T = nbx * dx, nby * dx
    row = np.arange(-1, nbx + 1)
    col = np.arange(nby)
    pts = np.concatenate([
        np.stack([(row + 0.5) * dx, np.full(row.size, -0.5 * dx)], axis=1),
        np.stack([(row + 0.5) * dx, np.full(row.size, T + 0.5 * dx)], axis=1),
        np.stack([np.full(col.size, -0.5 * dx), (col + 0.5) * dx], axis=1),
        np.stack([np.full(col.size, W + 0.5 * dx), (col + 0.5) * dx], axis=1)])
    boundary = _wall("boundary", pts, mass, c0, rho0)
    kernel = CubicSplineKernel(h, ndims=2)
    inters = [SystemInteraction(kernel, FluidPfn(alpha, beta, h), fluid),
              SystemInteraction(kernel, FluidPfn(alpha, beta, h), fluid, StaticBoundarySystem(boundary, dx))]
    lf = LeapFrogTimeIntegrator([fluid, boundary], inters)
    meta = dict(workload="dambreak_lj_2d", n_fluid=fluid.n, n_boundary=boundary.n, h=h, c0=c0, cfl=cfl,
                dt=cfl * h / c0, ndims=2)
    return lf, meta


def dambreak_lj_3d(nfx=50, nfy=12, nfz=50, nbx=150, nby=12, nbz=80, dx=0.5, rho0=1000.0, alpha=0.005, beta=0.0,
                   hfac=1.2, cfl=0.05, column_height=None):
    """3-D dam break in a single-layer Lennard-Jones box (dambreak_3d.jl
    layout, z vertical): an nfx×nfy×nfz block (i, j, m loops, m innermost)
    at rest, and six faces of wall particles in the script's order (floor
    and ceiling from -1 to nbx × -1 to nby, left and right nby×nbz, front
    and back nbx×nbz) in one BasicParticleSystem wrapped as
    StaticBoundarySystem(boundary, dx)."""
    H = nfz * dx if column_height is None else column_height
    c0 = 10.0 * math.sqrt(2.0 * G * H)
    h = hfac * dx
    mass = rho0 * dx ** 3
    ii, jj, mm = np.meshgrid(np.arange(nfx), np.arange(nfy), np.arange(nfz), indexing="ij")
    fluid = FluidParticleSystem("fluid", nfx * nfy * nfz, 3, mass, c0, source_v=[0.0, 0.0, -G],
                                state_updater=TaitEOSUpdater(rho0))
    fluid.x[:] = np.stack([(ii.ravel() + 0.5) * dx, (jj.ravel() + 0.5) * dx, (mm.ravel() + 0.5) * dx], axis=1)
    fluid.rho[:] = rho0
    fluid.p[:] = _tait_pressure(fluid.rho, rho0, c0, 7.0)
    X, Y, Z = nbx * dx, nby * dx, nbz * dx

    def face(a, b, fixed_axis, value):
        A, B = np.meshgrid(a, b, indexing="ij")
        cols = [None, None, None]
        free = [ax for ax in range(3) if ax != fixed_axis]
        cols[free[0]], cols[free[1]] = A.ravel(), B.ravel()
        cols[fixed_axis] = np.full(A.size, value)
        return np.stack(cols, axis=1)

    ex = (np.arange(-1, nbx + 1) + 0.5) * dx
    ey = (np.arange(-1, nby + 1) + 0.5) * dx
    iy = (np.arange(nby) + 0.5) * dx
    iz = (np.arange(nbz) + 0.5) * dx
    ix = (np.arange(nbx) + 0.5) * dx
    pts = np.concatenate([face(ex, ey, 2, -0.5 * dx), face(ex, ey, 2, Z + 0.5 * dx),
                          face(iy, iz, 0, -0.5 * dx), face(iy, iz, 0, X + 0.5 * dx),
                          face(ix, iz, 1, -0.5 * dx), face(ix, iz, 1, Y + 0.5 * dx)])
    boundary = _wall("boundary", pts, mass, c0, rho0)
    kernel = CubicSplineKernel(h, ndims=3)
    inters = [SystemInteraction(kernel, FluidPfn(alpha, beta, h), fluid),
              SystemInteraction(kernel, FluidPfn(alpha, beta, h), fluid, StaticBoundarySystem(boundary, dx))]
    lf = LeapFrogTimeIntegrator([fluid, boundary], inters)
    meta = dict(workload="dambreak_lj_3d", n_fluid=fluid.n, n_boundary=boundary.n, h=h, c0=c0, cfl=cfl,
                dt=cfl * h / c0, ndims=3)
    return lf, meta


# ---------------------------------------------------------- column collapse

def column_collapse(nx=400, ny=200, dx=0.0005, rho0=2650.0, E=0.84e6, nu=0.3, phi_deg=19.8, psi=0.0,
                    cohesion=0.0, alpha=0.1, beta=0.1, hfac=1.5, cfl=0.1, bottom_len=None, layers=3,
                    wall_beta=3.0, geostatic=True):
    """2-D granular column collapse with the elasto-plastic Drucker–Prager
    updater (EP_ColumnCollapse.jl layout): column nx×ny, dynamic bottom of
    `layers` rows, ghost-mirrored left wall at x=0 (cutoff 3h, stress copied
    at stage 1), stages (StrainRateVorticityPfn, CauchyFluidPfn)."""
    phi = phi_deg * math.pi / 180.0
    c = math.sqrt(E * (1 - nu) / (rho0 * (1 + nu) * (1 - 2 * nu)))
    h = hfac * dx
    mass = rho0 * dx * dx
    ii, jj = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    x = np.stack([(ii.ravel() + 0.5) * dx, (jj.ravel() + 0.5) * dx], axis=1)
    fluid = ElastoPlasticParticleSystem(
        "soil", len(x), 2, 4, mass, c, source_v=[0.0, -G],
        state_updater=(ZeroFieldUpdater("strain_rate", "vorticity"),
                       ElastoPlasticStressUpdater(E, nu, phi, psi, cohesion)))
    fluid.x[:] = x
    fluid.rho[:] = rho0
    if geostatic:
        Hc = ny * dx
        K0 = 1.0 - math.sin(phi)
        syy = -rho0 * G * (Hc - x[:, 1])
        fluid.stress[:, 0] = K0 * syy
        fluid.stress[:, 1] = syy
        fluid.stress[:, 2] = K0 * syy
    if bottom_len is None:
        bottom_len = max(2.5 * nx * dx, nx * dx + 20 * dx)
    nbx = int(round(bottom_len / dx))
    bx = np.array([((i - 3.5) * dx, -(j - 0.5) * dx) for i in range(1, nbx + 4) for j in range(1, layers + 1)])
    bottom = _wall("bottom", bx, mass, c, rho0)
    ghost = GhostParticleSystem(fluid, GhostCopier("stress"))
    gentry = GhostEntry(ghost, 3.0 * h, ((1.0, 0.0), (0.0, 0.0)), capacity=int(fluid.n))
    kernel = CubicSplineKernel(h, ndims=2)
    srv = StrainRateVorticityPfn()
    cau = CauchyFluidPfn(alpha, beta, h)
    dyn = DynamicBoundarySystem(bottom, (0.0, 1.0), (0.0, 0.0), wall_beta)
    inters = [SystemInteraction(kernel, (srv, cau), fluid),
              SystemInteraction(kernel, (srv, cau), fluid, dyn),
              SystemInteraction(kernel, (srv, cau), fluid, ghost)]
    lf = LeapFrogTimeIntegrator([fluid, bottom], inters, ghosts=(gentry,))
    meta = dict(workload="column_collapse", n_fluid=fluid.n, n_boundary=bottom.n, h=h, c0=c, cfl=cfl,
                dt=cfl * h / c, ndims=2, phi=phi, E=E)
    return lf, meta


def granular_column(nfx=100, nfy=50, dx=0.002, rho0=1850.0, E=0.84e6, nu=0.3, phi_deg=19.8, cohesion=0.0,
                    alpha=0.1, beta=0.1, delta=0.1, hfac=1.2, cfl=0.1, bottom_len=0.5, layers=3, wall_beta=3.0):
    """2-D granular column collapse with the visco-plastic Mohr–Coulomb
    updater (GranularColumnCollapse.jl layout): StressParticleSystem NS = 3,
    stages (StrainRatePfn, CauchyFluidPfn with δ-SPH), dynamic bottom, ghost
    left wall with the stress copied at stage 2, LinearEOS inside the stress
    updater."""
    phi = phi_deg * math.pi / 180.0
    c = math.sqrt(E * (1 - nu) / (rho0 * (1 + nu) * (1 - 2 * nu)))
    h = hfac * dx
    mass = rho0 * dx * dx
    ii, jj = np.meshgrid(np.arange(nfx), np.arange(nfy), indexing="ij")
    x = np.stack([(ii.ravel() + 0.5) * dx, (jj.ravel() + 0.5) * dx], axis=1)
    fluid = StressParticleSystem(
        "fluid", len(x), 2, 3, mass, c, source_v=[0.0, -G],
        state_updater=(ZeroFieldUpdater("strain_rate"),
                       ViscoPlasticMCStressUpdater(LinearEOSUpdater(rho0), phi, cohesion)))
    fluid.x[:] = x
    fluid.rho[:] = rho0
    nbx = int(math.floor(bottom_len / dx))
    bx = np.array([((i - 3.5) * dx, -(j - 0.5) * dx) for i in range(1, nbx + 4) for j in range(1, layers + 1)])
    bottom = _wall("bottom_boundary", bx, mass, c, rho0)
    ghost = GhostParticleSystem(fluid, None, GhostCopier("stress"))
    gentry = GhostEntry(ghost, 3.0 * h, ((1.0, 0.0), (0.0, 0.0)), capacity=int(fluid.n))
    kernel = CubicSplineKernel(h, ndims=2)
    sr = StrainRatePfn()
    cau = CauchyFluidPfn(alpha, beta, h, delta=delta)
    dyn = DynamicBoundarySystem(bottom, (0.0, 1.0), (0.0, 0.0), wall_beta)
    inters = [SystemInteraction(kernel, (sr, cau), fluid),
              SystemInteraction(kernel, (sr, cau), fluid, dyn),
              SystemInteraction(kernel, (sr, cau), fluid, ghost)]
    lf = LeapFrogTimeIntegrator([fluid, bottom], inters, ghosts=(gentry,))
    meta = dict(workload="granular_column", n_fluid=fluid.n, n_boundary=bottom.n, h=h, c0=c, cfl=cfl,
                dt=cfl * h / c, ndims=2, phi=phi, E=E)
    return lf, meta


# ------------------------------------- EP column with virtual-particle walls

def ep_column_virtual(dx=0.002, width=0.2, height=0.1, bottom_len=0.5, rho0=1850.0, E=0.84e6, nu=0.3,
                      phi_deg=19.8, psi=0.0, cohesion=0.0, alpha=0.1, beta=0.1, hfac=1.2, cfl=0.1,
                      bottom_v=None, geostatic=False):
    """2-D elasto-plastic column collapse with virtual-particle boundaries
    (EP_ColumnCollapse2.jl layout): ElastoPlasticParticleSystem NS = 4 with
    four stages (nothing / zero strain rate and vorticity / EP stress
    update / nothing), a 3-layer bottom and a 3-column left wall as
    VirtualParticleSystems over StressParticleSystem sources, filled by
    InterpolateFieldFn(:v, :rho) at stage 1 and (:stress) at stage 3 and
    normalised by VirtualNormUpdater at stages 2 and 4 (bottom: no-slip,
    left: free-slip).  `bottom_v` gives the bottom a prescribed velocity
    (then it also carries a PrescribedVelocityUpdater at stage 2);
    `geostatic` starts the column from K0 stress instead of the script's
    zero stress."""
    phi = phi_deg * math.pi / 180.0
    c = math.sqrt(E * (1 - nu) / (rho0 * (1 + nu) * (1 - 2 * nu)))
    h = hfac * dx
    mass = rho0 * dx * dx
    nfx, nfy, nbx = int(math.floor(width / dx)), int(math.floor(height / dx)), int(math.floor(bottom_len / dx))
    fluid = ElastoPlasticParticleSystem(
        "fluid", nfx * nfy, 2, 4, mass, c, source_v=[0.0, -G],
        state_updater=(None, ZeroFieldUpdater("strain_rate", "vorticity"),
                       ElastoPlasticStressUpdater(E, nu, phi, psi, cohesion), None))
    ii, jj = np.meshgrid(np.arange(nfx), np.arange(nfy), indexing="ij")
    fluid.x[:, 0] = (ii.ravel() + 0.5) * dx
    fluid.x[:, 1] = (jj.ravel() + 0.5) * dx
    fluid.rho[:] = rho0
    if geostatic:
        K0 = 1.0 - math.sin(phi)
        syy = -rho0 * G * (nfy * dx - fluid.x[:, 1])
        fluid.stress[:, 0] = K0 * syy
        fluid.stress[:, 1] = syy
        fluid.stress[:, 2] = K0 * syy
    bsrc = StressParticleSystem("bottom_boundary", 3 * (nbx + 3), 2, 4, mass, c)
    bsrc.x[:] = [((i - 3.5) * dx, -(j - 0.5) * dx) for i in range(1, nbx + 4) for j in range(1, 4)]
    bsrc.rho[:] = rho0
    lsrc = StressParticleSystem("left_boundary", 3 * nfy, 2, 4, mass, c)
    lsrc.x[:] = [(-(col - 0.5) * dx, (j + 0.5) * dx) for j in range(nfy) for col in range(1, 4)]
    lsrc.rho[:] = rho0
    norm_b = VirtualNormUpdater((-1.0, -1.0), "v", "rho")
    bottom = VirtualParticleSystem(
        bsrc, "bottom_virt", bsrc.n, 2, mass, c, zero_fields=("v", "rho", "stress"), prescribed_v=bottom_v,
        state_updater=(None, norm_b if bottom_v is None else (norm_b, PrescribedVelocityUpdater()), None,
                       VirtualNormUpdater((-1.0, -1.0), "stress")))
    left = VirtualParticleSystem(
        lsrc, "left_virt", lsrc.n, 2, mass, c, zero_fields=("v", "rho", "stress"),
        state_updater=(None, VirtualNormUpdater((-1.0, 1.0), "v", "rho"), None,
                       VirtualNormUpdater((-1.0, 1.0), "stress")))
    kernel = CubicSplineKernel(h, ndims=2)
    sr = StrainRateVorticityPfn()
    kin = CauchyFluidPfn(alpha, beta, h)
    iv = InterpolateFieldFn("v", "rho", accumulate_wsum=True)
    istr = InterpolateFieldFn("stress", accumulate_wsum=False)
    inters = [SystemInteraction(kernel, (None, sr, None, kin), fluid),
              SystemInteraction(kernel, (iv, sr, istr, kin), fluid, bottom),
              SystemInteraction(kernel, (iv, sr, istr, kin), fluid, left)]
    lf = LeapFrogTimeIntegrator([fluid], inters, virtual_systems=(bottom, left))
    meta = dict(workload="ep_column_virtual", n_fluid=fluid.n, n_bottom=bsrc.n, n_left=lsrc.n, h=h, c0=c,
                cfl=cfl, dt=cfl * h / c, ndims=2)
    return lf, meta


# ------------------------------------------------------------------ trapdoor

def trapdoor(nx=264, ny=100, ntd_x=40, n_layers=10, dx=0.05, rho0=1600.0, E=10.0e6, nu=0.33, phi_deg=39.0,
             psi_deg=19.0, cohesion=0.0, alpha=0.1, beta=0.0, moving=False, trapdoor_v=-0.005, damping=0.002,
             cfl=0.1, geostatic=False):
    """2-D trapdoor (Trapdoor.jl layout): an nx x ny ElastoPlasticParticleSystem
    soil (NS = 4, four stages), left and right free-slip walls as one
    GhostEntry whose ghosts copy the stress (Householder-reflected) at stage
    3, a static bottom on both flanks and a centre trapdoor of ntd_x columns
    as VirtualParticleSystems (n_layers layers below y = 0), filled by
    InterpolateFieldFn(:rho) at stage 1 and (:stress) at stage 3 from the
    soil and from the wall ghosts (ghost_bottom: the ghost system as
    system_a), normalised at stages 2 and 4, and five stress probes across
    the trapdoor's top.  `moving=False` is the script's settling integrator
    (trapdoor and probes static, damping Γ); `moving=True` its second
    integrator (trapdoor and probes at trapdoor_v, no damping).
    `geostatic` starts the soil from K0 stress instead of zero stress."""
    phi, psi = phi_deg * math.pi / 180.0, psi_deg * math.pi / 180.0
    c = math.sqrt(E * (1 - nu) / (rho0 * (1 + nu) * (1 - 2 * nu)))
    h = 1.2 * dx
    mass = rho0 * dx * dx
    nleft = (nx - ntd_x) // 2
    soil = ElastoPlasticParticleSystem(
        "soil", nx * ny, 2, 4, mass, c, source_v=[0.0, -G],
        state_updater=(None, ZeroFieldUpdater("strain_rate", "vorticity"),
                       ElastoPlasticStressUpdater(E, nu, phi, psi, cohesion), None))
    ii, jj = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")  # i outer, j inner
    soil.x[:, 0] = (ii.ravel() + 0.5) * dx
    soil.x[:, 1] = (jj.ravel() + 0.5) * dx
    soil.rho[:] = rho0
    if geostatic:
        K0 = 1.0 - math.sin(phi)
        syy = -rho0 * G * (ny * dx - soil.x[:, 1])
        soil.stress[:, 0] = K0 * syy
        soil.stress[:, 1] = syy
        soil.stress[:, 2] = K0 * syy
    flank = [i for i in range(-5, nleft)] + [i for i in range(nleft + ntd_x, nx + 5)]
    bpts = [((i + 0.5) * dx, -(j - 0.5) * dx) for j in range(1, n_layers + 1) for i in flank]
    bsrc = StressParticleSystem("bottom_source", len(bpts), 2, 4, mass, c)
    bsrc.x[:] = bpts
    bsrc.rho[:] = rho0
    tpts = [((i + 0.5) * dx, -(j - 0.5) * dx) for j in range(1, n_layers + 1) for i in range(nleft, nleft + ntd_x)]
    tsrc = StressParticleSystem("trapdoor_source", len(tpts), 2, 4, mass, c)
    tsrc.x[:] = tpts
    tsrc.rho[:] = rho0
    upd = (None, (VirtualNormUpdater((0.0, 0.0), "rho"), PrescribedVelocityUpdater()), None,
           VirtualNormUpdater((0.0, 0.0), "stress"))
    bottom = VirtualParticleSystem(bsrc, "bottom_virt", bsrc.n, 2, mass, c, zero_fields=("v", "rho", "stress"),
                                   state_updater=upd)
    pv = (0.0, trapdoor_v) if moving else None
    door = VirtualParticleSystem(tsrc, "trapdoor_moving_virt" if moving else "trapdoor_static_virt", tsrc.n, 2,
                                 mass, c, zero_fields=("v", "rho", "stress"), prescribed_v=pv, state_updater=upd)
    ghost = GhostParticleSystem(soil, None, None, GhostCopier(("stress", HouseholderReflect())), None,
                                name="walls_ghost")
    walls = GhostEntry(ghost, 3.0 * h, ((1.0, 0.0), (0.0, 0.0)), ((-1.0, 0.0), (nx * dx, 0.0)))
    kernel = CubicSplineKernel(h, ndims=2)
    sr = StrainRateVorticityPfn()
    kin = CauchyFluidPfn(alpha, beta, h)
    irho = InterpolateFieldFn("rho", accumulate_wsum=True)
    istr = InterpolateFieldFn("stress", accumulate_wsum=False)
    inters = [SystemInteraction(kernel, (None, sr, None, kin), soil),
              SystemInteraction(kernel, (irho, sr, istr, kin), soil, bottom),
              SystemInteraction(kernel, (irho, None, istr, None), ghost, bottom),
              SystemInteraction(kernel, (irho, sr, istr, kin), soil, door),
              SystemInteraction(kernel, (None, sr, None, kin), soil, ghost)]
    npr = 5
    ppos = [(nleft * dx + k * (ntd_x * dx / (npr - 1)), 0.0) for k in range(npr)]
    probe = ProbeParticleSystem("td_probe_moving" if moving else "td_probe_static", ppos,
                                extras={"stress": np.zeros((npr, 4))},
                                state_updater=VirtualNormUpdater((1.0, 1.0), "stress"), prescribed_v=pv)
    pint = SystemInteraction(kernel, InterpolateFieldFn("stress"), soil, probe)
    kw = {} if moving else {"Γ": damping}
    lf = LeapFrogTimeIntegrator([soil], inters, ghosts=(walls,), virtual_systems=(bottom, door), probes=(probe,),
                                probe_interactions=(pint,), **kw)
    meta = dict(workload="trapdoor", n_soil=soil.n, n_bottom=bsrc.n, n_trapdoor=tsrc.n, h=h, c0=c, cfl=cfl,
                dt=cfl * h / c, ndims=2)
    return lf, meta


# ------------------------------------------------ dam break on an elastic wall

def dambreak_wall(dx=0.5, nfx=50, nfy=50, cfl=0.05, x_wall=60.0):
    """2-D dam break against a linear-elastic wall (DambreakWall.jl layout):
    a 25 m x 25 m water column (Tait at stage 2), a 1.5 m x 10 m
    ElastoPlasticParticleSystem wall (NS = 4, StrainRateVorticityPfn then
    CauchyFluidPfn, Hooke stress update) standing on the floor at x = 60 m,
    FluidSolidPfn from the water onto the wall, and four 3-layer dynamic
    boundaries (floor, left, right, top).  `dx` scales the spacing; the
    particle counts follow the script's extents; `x_wall` moves the wall
    (next to the column, the fluid loads it from the first step)."""
    g = (0.0, -9.81)
    rho_w, c = 1000.0, 10.0 * math.sqrt(2.0 * 9.81 * 25.0)
    alpha, beta = 0.02, 0.0
    rho_s, E, nu = 2400.0, 5.0e8, 0.2
    c_s = math.sqrt(E * (1 - nu) / (rho_s * (1 + nu) * (1 - 2 * nu)))
    h = 1.2 * dx
    fm = rho_w * dx * dx
    fluid = FluidParticleSystem("fluid", nfx * nfy, 2, fm, c, source_v=g,
                                state_updater=(None, TaitEOSUpdater(rho_w)))
    jj, ii = np.meshgrid(np.arange(nfy), np.arange(nfx), indexing="ij")
    fluid.x[:, 0] = (ii.ravel() + 0.5) * dx
    fluid.x[:, 1] = (jj.ravel() + 0.5) * dx
    fluid.rho[:] = rho_w
    fluid.p[:] = _tait_pressure(fluid.rho, rho_w, c, 7.0)  # update_state!(fluid, 2)
    nwx, nwy = int(round(1.5 / dx)), int(round(10.0 / dx))
    wall = ElastoPlasticParticleSystem("wall", nwx * nwy, 2, 4, rho_s * dx * dx, c_s, source_v=g,
                                       state_updater=(ZeroFieldUpdater("strain_rate", "vorticity"),
                                                      HookeLawStressUpdater(E, nu)))
    jj, ii = np.meshgrid(np.arange(nwy), np.arange(nwx), indexing="ij")
    wall.x[:, 0] = x_wall + (ii.ravel() + 0.5) * dx
    wall.x[:, 1] = (jj.ravel() + 0.5) * dx
    wall.rho[:] = rho_s
    x_right, y_top, layers = 75.0, 40.0, 3
    nfl = int(round((76.25 + 1.25) / dx)) + 1
    nly = int(round(40.0 / dx))

    def layer_sys(name, pts):
        ps = BasicParticleSystem(name, len(pts), 2, fm, c)
        ps.x[:] = pts
        ps.rho[:] = rho_w
        return ps

    floor = layer_sys("floor", np.array([(-1.25 + ix * dx, -(ly + 0.5) * dx)
                                         for ly in range(layers) for ix in range(nfl)]))
    left = layer_sys("left", np.array([(-(ly + 0.5) * dx, (iy + 0.5) * dx)
                                       for ly in range(layers) for iy in range(nly)]))
    right = layer_sys("right", np.array([(x_right + (ly + 0.5) * dx, (iy + 0.5) * dx)
                                         for ly in range(layers) for iy in range(nly)]))
    top = layer_sys("top", np.array([(-1.25 + ix * dx, y_top + (ly + 0.5) * dx)
                                     for ly in range(layers) for ix in range(nfl)]))
    floor_d = DynamicBoundarySystem(floor, (0.0, 1.0), (0.0, 0.0), 3.0)
    left_d = DynamicBoundarySystem(left, (1.0, 0.0), (0.0, 0.0), 3.0)
    right_d = DynamicBoundarySystem(right, (-1.0, 0.0), (x_right, 0.0), 3.0)
    top_d = DynamicBoundarySystem(top, (0.0, -1.0), (0.0, y_top), 3.0)
    kernel = CubicSplineKernel(h, ndims=2)
    fpfn = FluidPfn(alpha, beta, h)
    cau = CauchyFluidPfn(alpha, beta, h)
    srv = StrainRateVorticityPfn()
    inters = [SystemInteraction(kernel, (None, fpfn), fluid),
              SystemInteraction(kernel, (srv, cau), wall),
              SystemInteraction(kernel, (None, FluidSolidPfn(alpha, beta, h)), fluid, wall),
              SystemInteraction(kernel, (None, fpfn), fluid, floor_d),
              SystemInteraction(kernel, (None, fpfn), fluid, left_d),
              SystemInteraction(kernel, (None, fpfn), fluid, right_d),
              SystemInteraction(kernel, (None, fpfn), fluid, top_d),
              SystemInteraction(kernel, (srv, cau), wall, floor_d)]
    lf = LeapFrogTimeIntegrator([fluid, wall, floor, left, right, top], inters)
    meta = dict(workload="dambreak_wall", n_fluid=fluid.n, n_wall=wall.n, h=h, c0=max(c, c_s), cfl=cfl, ndims=2)
    return lf, meta


# ------------------------------------------------------- multiphase bubble

BUBBLE_VARIANTS = {
    # rho_Y, c_Y / sqrt(g R), gamma_Y, sigma, epsilon (X-Y), XSPH epsilon, dx
    "bubble": (500.0, 40.0, 7.0, 2, None, None, 0.05),
    "bubble2": (10.0, math.sqrt(16000.0), 1.4, 1, None, None, 0.04),
    "bubble3": (1.0, 400.0, 1.4, 1, 0.1, 0.5, 0.04),
}


def bubble(variant="bubble", R=1.0, dx=None, rho_x=1000.0, alpha=0.01, beta=0.0, hfac=1.2, cfl=1.5,
           integrator="rk4", xsph=True):
    """2-D light-fluid bubble rising in a heavy fluid (bubble.jl /
    bubble2.jl / bubble3.jl layout): a 6R x 10R column of fluid X with a
    disc of radius R of fluid Y centred at the origin, both Tait fluids with
    hydrostatic initial density and zero initial pressure, Wendland C2
    kernel, FluidPfn self interactions, the two-sided X-Y FluidPfn with Y
    first, a one-stage ghost of X with its pressure copied, mirrored across
    the four walls and the four diagonal corner planes.  bubble3 adds
    XSPHPfn(0.5) velocity adjustment on X, Y and X-ghost (`xsph=False`
    leaves it out)."""
    rho_y, cy_fac, gamma_y, sigma, eps, xeps, dx0 = BUBBLE_VARIANTS[variant]
    xs = XSPHPfn(xeps) if (xsph and xeps is not None) else None
    dx = dx0 if dx is None else dx
    height, width = 10.0 * R, 6.0 * R
    y_min, x_min = -2.0 * R, -3.0 * R
    y_max, x_max = y_min + height, x_min + width
    h = hfac * dx
    c_x = math.sqrt(800.0 * G * R)
    c_y = cy_fac * math.sqrt(G * R)
    nx, ny = int(math.floor(width / dx)), int(math.floor(height / dx))
    ii, jj = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    px = x_min + (ii.ravel() + 0.5) * dx
    py = y_min + (jj.ravel() + 0.5) * dx
    inside = px * px + py * py < R * R
    systems = []
    for name, sel, rho0, c, gamma in (("fluid X", ~inside, rho_x, c_x, 7.0),
                                       ("fluid Y", inside, rho_y, c_y, gamma_y)):
        n = int(sel.sum())
        ps = FluidParticleSystem(name, n, 2, dx * dx * rho0, c, source_v=[0.0, -G],
                                 state_updater=TaitEOSUpdater(rho0, gamma))
        ps.x[:, 0] = px[sel]
        ps.x[:, 1] = py[sel]
        pressure = (y_min + height - ps.x[:, 1]) * rho_x * G
        ps.rho[:] = (pressure * gamma / (c * c * rho0) + 1.0) ** (1.0 / gamma) * rho0
        systems.append(ps)
    fx, fy = systems
    ghost = GhostParticleSystem(fx, GhostCopier("p"), name="ghost[fluid_X]")
    s2 = 1.0 / math.sqrt(2.0)
    gentry = GhostEntry(ghost, 3.0 * h,
                        ((1.0, 0.0), (x_min, 0.0)), ((-1.0, 0.0), (x_max, 0.0)),
                        ((0.0, 1.0), (0.0, y_min)), ((0.0, -1.0), (0.0, y_max)),
                        ((s2, s2), (x_min, y_min)), ((-s2, s2), (x_max, y_min)),
                        ((s2, -s2), (x_min, y_max)), ((-s2, -s2), (x_max, y_max)))
    kernel = WenlandC2Kernel(h, ndims=2)
    pfn = FluidPfn(alpha, beta, h, sigma=sigma)
    inters = [SystemInteraction(kernel, pfn, fx, velocity_adjust_pairwise_fn=xs),
              SystemInteraction(kernel, pfn, fy, velocity_adjust_pairwise_fn=xs),
              SystemInteraction(kernel, FluidPfn(alpha, beta, h, sigma=sigma, epsilon=eps), fy, fx),
              SystemInteraction(kernel, pfn, fx, ghost, velocity_adjust_pairwise_fn=xs)]
    cls = RK4TimeIntegrator if integrator == "rk4" else LeapFrogTimeIntegrator
    lf = cls([fx, fy], inters, ghosts=(gentry,))
    meta = dict(workload=variant, n_fluid=fx.n + fy.n, n_x=fx.n, n_y=fy.n, h=h, c0=max(c_x, c_y), cfl=cfl,
                ndims=2)
    return lf, meta


def batched_columns(count=256, seed=20261203, nmin=2000, nmax=60000, dx=0.0005, **kw):
    """`count` column collapses with log-uniform particle counts, aspect
    ratio H/W ~ U[0.5, 4], friction angle ~ U[25°, 40°], E ~ U[0.5, 5] MPa."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        N = math.exp(rng.uniform(math.log(nmin), math.log(nmax)))
        ar = rng.uniform(0.5, 4.0)
        nx = max(2, int(round(math.sqrt(N / ar))))
        ny = max(2, int(round(N / nx)))
        phi = rng.uniform(25.0, 40.0)
        E = rng.uniform(0.5e6, 5.0e6)
        out.append(column_collapse(nx=nx, ny=ny, dx=dx, phi_deg=phi, E=E, **kw))
    return out
