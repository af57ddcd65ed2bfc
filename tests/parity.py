"""The per-particle error metric of the parity tests.

The device and the oracle evaluate the same pair terms (bit-identical in
FP64; FP32 in the compensated mode) but sum each particle's terms in a
different order: the device gathers them per particle, the reference
scatters them in colour order.  A rate field that cancels to near zero
(dv/dt of a particle in hydrostatic balance starts at gravity and loses it
to the pressure terms) therefore differs by a few ulps of its terms, not of
its value.  The error of particle i, component k, is measured against

* rate fields (dvdt, drhodt, strain_rate, vorticity):
  ``max(|ref_ik|, M_ik)`` where ``M_ik`` is the oracle's magnitude shadow:
  |initial value| + Σ|every term added since| (``track_magnitude``);
* v, rho and x, integrated from the rates: ``max(|q_ik|, I_ik)`` where
  ``I_ik`` is the oracle's integrated shadow, Σ over the steps since the
  upload of each increment's magnitude (dt·M of the rate; for x,
  dt·max(|v|, I(v)));
* p: ``max(|p_i|, c²·I(rho)_i)`` for equation-of-state systems (the
  pressure of the density increments; dp/dρ = c² for the linear EOS and
  near ρ0 for Tait), the particle's stress norm for stress systems; a
  stress set from the pressure (visco-plastic Mohr-Coulomb) takes three
  times the pressure's scale as a floor;
* stress: ``max(max_k |σ_ik|, max_k I(σ)_ik)``, the particle's tensor
  max-norm or the summed magnitude of its stress increments (the oracle's
  dt·|D|·M(ε̇) + 2·dt·|σ|·M(ω) per step), whichever is larger; strain and
  plastic strain: the max-norm over both tensors of the particle or the
  summed magnitude of its strain increments (dt·M(ε̇) per step).

After many steps a pressure is compared in density units, on
``max(|p_i|, c²·scale(rho)_i)`` (and the stress scale of a stress system):
an equation-of-state p is a function of ρ alone (dp/dρ = c² for the linear
EOS, ≈ c² near ρ0 for Tait), and a pressure at round-off level around zero
(a free-falling column) would otherwise be judged against itself.

Each scale is then taken per particle over the field's components (the
largest component scale of the particle's vector or tensor): a velocity's x
component in a free-falling column is round-off noise around zero, and is
judged against the particle's speed, not against itself.

A zero scale demands exact equality.  Particles are matched by id, so
comparisons after many steps do not depend on both sides sorting alike.

Two kinds of shadow (the oracle's magnitude modes):

* TERMS (mode 1), for one step from identical inputs: Σ|term| as above.
  The two sides evaluate bit-identical FP64 terms and differ only in the
  order of the sums.
* INPUTS (mode 2), for comparisons whose inputs differ: after many steps
  (the trajectories drifted by a few ulps) and for the FP32-compensated
  mode (its records round v, ρ, p/ρ² and σ to FP32).  Each term's
  magnitude is taken with every difference of its inputs replaced by the
  sum of their magnitudes (|v_i| + |v_j| for v_i - v_j, |ρ_i| + |ρ_j|,
  |p|, |σ|, |∇W| componentwise): a strain rate's (v_j - v_i)·∇W of a column
  at rest is far smaller than its inputs, and its error follows the inputs.

After many steps the rate fields are compared through
`one_step_from_device_state`: the device's state is handed to the oracle and
one further step compared on the TERMS scale.
"""
from __future__ import annotations

import numpy as np

TERMS, INPUTS = 1, 2

RATES = ("dvdt", "drhodt", "strain_rate", "vorticity")
_SHADOWED = {"x": 0, "v": 1, "rho": 2, "dvdt": 3, "drhodt": 4, "stress": 6, "strain_rate": 7, "vorticity": 8,
             "strain": 9}


def oracle_magnitudes(sess, lf, inst=0):
    """{system name: {rate field: magnitude shadow}} of an oracle session
    whose backend tracks magnitudes, in the systems' current order."""
    m = sess.maps[inst]
    out = {}
    for ps in m.systems:
        d = {}
        for name, fid in ps.particle_fields():
            if name in _SHADOWED:
                buf = np.zeros(np.shape(getattr(ps, name)))
                d[name] = sess.backend.magnitude(m.inst, m.h(ps), fid, buf)
        out[id(ps)] = d
    return out


def _col(a):
    a = np.asarray(a, dtype=float)
    return a.reshape(a.shape[0], -1) if a.ndim else a


def particle_scales(sc, mags, p_density_units=False):
    """Per-particle, per-component scales of every compared field of the
    reference system `sc`, from its magnitude shadows `mags`."""
    sc_f = {name: _col(getattr(sc, name)) for name, _ in sc.particle_fields() if name != "id"}
    out = {}
    for r in RATES:
        if r in sc_f:
            out[r] = np.maximum(np.abs(sc_f[r]), _col(mags[r]) if r in mags else 0.0)
    for q in ("x", "v", "rho"):
        if q in sc_f:
            out[q] = np.maximum(np.abs(sc_f[q]), _col(mags[q]) if q in mags else 0.0)
    if "v" in out:
        # XSPH's velocity adjustment is a correction of v, on v's scale
        out["v_adjustment"] = out["v"]
    if "stress" in sc_f:
        norm = np.abs(sc_f["stress"]).max(axis=1, keepdims=True)
        if "stress" in mags:
            norm = np.maximum(norm, _col(mags["stress"]).max(axis=1, keepdims=True))
        out["stress"] = np.broadcast_to(norm, sc_f["stress"].shape)
    if "p" in sc_f:
        floor = out["rho"] if p_density_units else _col(mags["rho"])
        p_eos = sc.c * sc.c * floor
        out["p"] = np.maximum(np.abs(sc_f["p"]), p_eos)
        if "stress" in sc_f:
            if _stress_from_pressure(sc):
                # σ = 2(c + p·tanφ)·ε̇/|ε̇| - p: |σ| ≤ 3|p| for φ ≤ 45°
                out["stress"] = np.maximum(out["stress"], 3.0 * p_eos[:, :1])
            out["p"] = np.maximum(out["p"] if p_density_units else np.abs(sc_f["p"]), out["stress"][:, :1])
    if "strain" in sc_f:
        norm = np.maximum(np.abs(sc_f["strain"]).max(axis=1, keepdims=True),
                          np.abs(sc_f["strain_p"]).max(axis=1, keepdims=True))
        if "strain" in mags:
            norm = np.maximum(norm, _col(mags["strain"]).max(axis=1, keepdims=True))
        out["strain"] = np.broadcast_to(norm, sc_f["strain"].shape)
        out["strain_p"] = out["strain"]
    # per particle: the largest component scale of the vector or tensor
    for name, a in out.items():
        a = np.asarray(a)
        if a.ndim == 2 and a.shape[1] > 1:
            out[name] = np.broadcast_to(a.max(axis=1, keepdims=True), a.shape)
    return out


def _errors(a, b, scale):
    a, b, scale = _col(a), _col(b), np.asarray(scale, dtype=float)
    d = np.abs(a - b)
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.where(scale > 0, d / np.where(scale > 0, scale, 1.0), np.where(d > 0, np.inf, 0.0))


def _stress_from_pressure(ps):
    """True when a system's stress is set algebraically from its
    equation-of-state pressure each step (the visco-plastic Mohr-Coulomb
    updater, src/StateUpdaters.jl:144-186), not integrated."""
    from grasph_b200.model import ViscoPlasticMCStressUpdater
    for entry in getattr(ps, "state_updater", ()):
        chain = entry if isinstance(entry, tuple) else (entry,)
        if any(isinstance(u, ViscoPlasticMCStressUpdater) for u in chain):
            return True
    return False


def field_error(a, b, scale):
    """max over particles and components of |a-b|/scale (0/0 = 0, x/0 = inf)."""
    e = _errors(a, b, scale)
    return float(e.max()) if e.size else 0.0


def _worst(a, b, scale, ids):
    """Where the largest error sits: particle id, component, both values
    and the scale (for the assertion message)."""
    e = _errors(a, b, scale)
    i, k = np.unravel_index(int(np.argmax(e)), e.shape)
    a, b, scale = _col(a), _col(b), np.broadcast_to(np.asarray(scale, dtype=float), e.shape)
    return f"id {int(ids[i])} comp {k}: device {a[i, k]:.17g} oracle {b[i, k]:.17g} scale {scale[i, k]:.3e}"


def _tol(tol, name):
    if isinstance(tol, dict):
        return tol.get(name, tol["*"])
    return tol


def compare_system(sg, sc, mags, tol, rate_tol=None, exact_ids=True, skip=(), report=None, p_density_units=None):
    """Assert every field of the device system `sg` within `tol` (a number,
    or {field: tolerance, "*": default}; rates: `rate_tol`, default `tol`)
    of the oracle system `sc` on the per-particle scales.  `exact_ids`: the
    two must also be in the same order (else matched by id, and an EOS
    pressure compared in density units unless `p_density_units` says
    otherwise).  Returns {field: error}."""
    if p_density_units is None:
        p_density_units = not exact_ids
    ig, ic = np.asarray(sg.id), np.asarray(sc.id)
    if exact_ids:
        assert np.array_equal(ig, ic), f"{sg.name}: permutation differs ({np.sum(ig != ic)} positions)"
        og = oc = slice(None)
    else:
        og, oc = np.argsort(ig, kind="stable"), np.argsort(ic, kind="stable")
        assert np.array_equal(ig[og], ic[oc]), f"{sg.name}: particle ids differ"
    scales = particle_scales(sc, mags, p_density_units)
    errs = {}
    for name, _ in sg.particle_fields():
        if name == "id" or name in skip:
            continue
        a = _col(getattr(sg, name))[og]
        b = _col(getattr(sc, name))[oc]
        s = np.asarray(scales[name])[oc]
        e = field_error(a, b, s)
        errs[name] = e
        t = rate_tol if (rate_tol is not None and name in RATES) else _tol(tol, name)
        assert e <= t, f"{sg.name}.{name}: per-particle error {e:.3e} exceeds {t} ({_worst(a, b, s, ic[oc])})"
    if report is not None:
        report[sg.name] = errs
    return errs


def compare_integrators(lf_g, lf_c, sess_c, tol, rate_tol=None, exact_ids=True, skip=(), report=None):
    """compare_system over every system of two integrators built alike."""
    mags = oracle_magnitudes(sess_c, lf_c)
    out = {}
    for sg, sc in zip(lf_g.systems, lf_c.systems):
        out[sg.name] = compare_system(sg, sc, mags[id(sc)], tol, rate_tol, exact_ids, skip, report)
    return out


def copy_state(lf_from, lf_to):
    """Every field of every system of `lf_from` into the alike-built `lf_to`."""
    for a, b in zip(lf_from.systems, lf_to.systems):
        for name, _ in a.particle_fields():
            getattr(b, name)[...] = getattr(a, name)


def one_step_from_device_state(lf_g, lf_c, g, c, cfl, tol, rate_tol=None, skip=(), report=None, mode=TERMS):
    """The device's current state (pulled into `lf_g`) handed to the oracle
    session `c`; one further step on both; every field compared on the
    per-particle scale (the oracle's shadows in `mode`) with the
    permutation bit-exact."""
    copy_state(lf_g, lf_c)
    c.backend.set_track_magnitude(mode)
    c.push()
    g.step(1, cfl)
    c.step(1, cfl)
    g.pull()
    c.pull()
    return compare_integrators(lf_g, lf_c, c, tol, rate_tol, exact_ids=True, skip=skip, report=report)


def run_and_compare(builder, nsteps, cfl, tol, precision=None, rate_tol=None, threads=1, one_step_tol=1e-10):
    """Build the scenario twice (`builder()` returns an integrator, or an
    (integrator, meta) pair), run `nsteps` on the device (FP64, or
    `precision`) and on the magnitude-tracking oracle, and compare:
    after one step every field at `tol` (rates at `rate_tol`); after more,
    the state on its integrated scale at `tol`, then (FP64 only) one further
    step from the device's state at `one_step_tol`.  The oracle's shadows
    are over the pair terms for one FP64 step and over the inputs otherwise.
    Returns the device and oracle integrators and sessions."""
    import grasph_b200 as G
    from gc_helpers import make_backend

    def build():
        r = builder()
        return r[0] if isinstance(r, tuple) else r

    lf_g, lf_c = build(), build()
    prec = G.PRECISION_FP64 if precision is None else precision
    mode = one_step_mode(lf_g, prec) if nsteps == 1 else INPUTS
    g = G.Session([lf_g], backend=make_backend("cuda"), precision=prec)
    c = G.Session([lf_c], backend=make_backend("oracle", track=mode, threads=threads))
    for s in (g, c):
        s.push()
        s.step(nsteps, cfl)
        s.pull()
    if nsteps == 1:
        compare_integrators(lf_g, lf_c, c, tol, rate_tol)
    else:
        compare_integrators(lf_g, lf_c, c, tol, exact_ids=False, skip=RATES)
        if prec == G.PRECISION_FP64:
            one_step_from_device_state(lf_g, lf_c, g, c, cfl, one_step_tol, mode=one_step_mode(lf_g, prec))
    return lf_g, lf_c, g, c


def one_step_mode(lf, precision):
    """The shadow kind for one step from identical inputs: TERMS for a FP64
    LeapFrog step (one evaluation of the pair terms); INPUTS for the
    compensated mode and for RK4, whose later right-hand-side evaluations
    start from intermediate states that already differ by the first ones'
    summation order."""
    import grasph_b200 as G
    from grasph_b200 import consts as C
    if precision != G.PRECISION_FP64 or getattr(lf, "kind", C.GC_INTEGRATOR_LEAPFROG) != C.GC_INTEGRATOR_LEAPFROG:
        return INPUTS
    return TERMS
