"""Error of the mixed-precision engine against the FP64 engine.

The FP64 engine reproduces the reference solver's V to 1e-12 (its parity tests
against the reference's own code), so it is the comparator for the mixed form
at lattice sizes the CPU cannot run.  ``compare_mixed_fp64`` evolves the same
events (same seeds, MV initial conditions, couplings and step counts) through
both engines on the GPU, measures each event's dipole correlator once at the
end (lfield::trace + gfield::average_and_symmetrize, field.h:1375-1492) and
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


def _run(jw, precision: int, specs, device: int, reunitarize: bool):
    eng = jw.Engine(precision=precision, device=device, reunitarize=reunitarize)
    ids = [eng.add_event(s["N"], ny_slices=s["ny_slices"], mu=s["mu"], mass=s["mass"], step=s["step"],
                         coupling=s["coupling"], seed=s["seed"]) for s in specs]
    eng.init_mv(ids)
    for eid, s in zip(ids, specs):
        eng.step([eid], s["steps"])
    eng.measure(ids)
    out = []
    for eid in ids:
        Sb, rb, cb, qs = eng.dipole(eid)
        out.append(dict(S=Sb, r=rb, Qs=qs, drift=_drift(eng.get_V(eid))))
    status = eng.sync()
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
