"""Error of the mixed-precision engine against the FP64 engine.

The FP64 engine reproduces the reference solver's V to 1e-12 (its parity tests
against the reference's own code), so it is the comparator for the mixed form
at lattice sizes the CPU cannot run; above its largest size (1024^2) the
call-for-call FP64 layer, pinned to the reference the same way, takes its
place.  ``compare_mixed_fp64`` evolves the same events (same seeds, MV
initial conditions, couplings and step counts) in FP64 and in mixed precision
on the GPU, measures each event's dipole correlator once at the end (lfield::trace + gfield::average_and_symmetrize, field.h:1375-1492) and
reports, per event and for the ensemble mean:

* max |S_mixed(r) - S_fp64(r)| over the angle-averaged bins,
* |Q_s,mixed - Q_s,fp64| / Q_s,fp64,
* the unitarity drift max |V V^dagger - 1| of the mixed V (and of the FP64 V).

S(r) and Q_s follow the library's definition (jw_engine_dipole): S(r) is the
angular average of (1/3N^2) sum_x tr V(x) V^dagger(x + r) over bins
b = floor(|r| + 1/2), and Q_s = sqrt(2)/r_s with S(r_s) = exp(-1/2),
interpolated linearly between the first pair of bins that brackets it.
"""
from __future__ import annotations

import math

import numpy as np


def qs_from_bins(S: np.ndarray, r: np.ndarray) -> float:
    """Q_s of angle-averaged bins, the same rule as jw_engine_dipole."""
    target = math.exp(-0.5)
    for b in range(len(S) - 1):
        if S[b] >= target and S[b + 1] < target:
            t = (S[b] - target) / (S[b] - S[b + 1])
            rs = r[b] + t * (r[b + 1] - r[b])
            return math.sqrt(2.0) / rs if rs > 0 else 0.0
    return 0.0


def _drift(V: np.ndarray) -> float:
    M = V.reshape(-1, 3, 3)
    return float(np.abs(M @ np.conj(np.transpose(M, (0, 2, 1))) - np.eye(3)).max())


FP64_ENGINE_MAX_N = 1024  # the FP64 engine's row pass holds 8 FP64 planes of a row


def _run_call_for_call(jw, s, device: int):
    """One event through the call-for-call FP64 layer (jw_initial_condition,
    jw_evolve_momentum, then execute2D + trace + average_and_symmetrize +
    jw_dipole), the comparator above the FP64 engine's largest size.  The
    noise stream is keyed by (seed, step) exactly as in the engine."""
    N = s["N"]
    ctx = jw.Context(jw.config_defaults(Nx=N, Ny=N, seed=s["seed"], mu=s["mu"], mass=s["mass"],
                                        elementaryWilsonLines=s["ny_slices"], step=s["step"],
                                        CouplingChoice=s["coupling"]), device)
    V, Vk, c = ctx.field(), ctx.field(), ctx.field(1)
    ctx.initial_condition(V)
    ctx.evolve_momentum(V, 0, s["steps"])
    Vk.copy_from(V)
    ctx.execute2D(Vk, 1)
    ctx.trace(Vk, c)
    ctx.average_and_symmetrize(c)
    Sb, rb, _, qs = ctx.dipole(c)
    out = dict(S=Sb, r=rb, Qs=qs, drift=_drift(V.get()))
    status = ctx.sync()
    ctx.close()
    return out, status


def _run(jw, precision: int, specs, device: int, reunitarize: bool):
    out = [None] * len(specs)
    status = jw.OK
    if precision == jw.PRECISION_FP64:
        for i, s in enumerate(specs):
            if s["N"] > FP64_ENGINE_MAX_N:
                out[i], st = _run_call_for_call(jw, s, device)
                status = status or st
    todo = [i for i in range(len(specs)) if out[i] is None]
    if todo:
        eng = jw.Engine(precision=precision, device=device, reunitarize=reunitarize)
        ids = [eng.add_event(specs[i]["N"], ny_slices=specs[i]["ny_slices"], mu=specs[i]["mu"],
                             mass=specs[i]["mass"], step=specs[i]["step"], coupling=specs[i]["coupling"],
                             seed=specs[i]["seed"]) for i in todo]
        eng.init_mv(ids)
        for eid, i in zip(ids, todo):
            eng.step([eid], specs[i]["steps"])
        eng.measure(ids)
        for eid, i in zip(ids, todo):
            Sb, rb, cb, qs = eng.dipole(eid)
            out[i] = dict(S=Sb, r=rb, Qs=qs, drift=_drift(eng.get_V(eid)))
        status = status or eng.sync()
        eng.close()
    return out, status


def compare_mixed_fp64(jw, specs, device: int = 0, reunitarize_mixed: bool = True) -> dict:
    """Evolve `specs` (dicts with N, ny_slices, mu, mass, step, coupling, seed,
    steps) in FP64 and in mixed precision and compare their dipoles.

    The mixed engine reunitarises V after every step (reunitarize_mixed), as
    the mixed form prescribes; the FP64 engine runs as the reference does,
    without reunitarisation.  Events of one lattice size form the ensemble
    whose mean S(r) is compared as well."""
    ref, st64 = _run(jw, jw.PRECISION_FP64, specs, device, False)
    mix, st32 = _run(jw, jw.PRECISION_MIXED, specs, device, reunitarize_mixed)
    per_event = []
    for s, a, b in zip(specs, mix, ref):
        dS = float(np.abs(a["S"] - b["S"]).max())
        dq = abs(a["Qs"] - b["Qs"]) / b["Qs"] if b["Qs"] > 0 else 0.0
        per_event.append(dict(N=s["N"], steps=s["steps"], coupling=s["coupling"], dS_max=dS, Qs=b["Qs"],
                              Qs_rel_err=dq, drift_mixed=a["drift"], drift_fp64=b["drift"]))
    ensembles = {}
    for n in sorted({s["N"] for s in specs}):
        idx = [i for i, s in enumerate(specs) if s["N"] == n]
        Sm = np.mean([mix[i]["S"] for i in idx], axis=0)
        Sf = np.mean([ref[i]["S"] for i in idx], axis=0)
        r = ref[idx[0]]["r"]
        qm, qf = qs_from_bins(Sm, r), qs_from_bins(Sf, r)
        ensembles[n] = dict(events=len(idx), dS_max=float(np.abs(Sm - Sf).max()), Qs=qf,
                            Qs_rel_err=abs(qm - qf) / qf if qf > 0 else 0.0)
    return dict(status=(st64, st32), per_event=per_event, ensembles=ensembles,
                dS_max=max(e["dS_max"] for e in per_event),
                Qs_rel_err_max=max(e["Qs_rel_err"] for e in per_event),
                drift_mixed_max=max(e["drift_mixed"] for e in per_event),
                drift_fp64_max=max(e["drift_fp64"] for e in per_event))
