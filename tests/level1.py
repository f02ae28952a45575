"""The level-1 bound shared by the GPU kernel tests and the CPU check of the
reference's own FP32 outputs (see the comment below)."""
import numpy as np

# Level-1 bound (north star): every finite BSDF / sampling / MIS output within 1e-5
# relative of the FP64 transcription of the reference's formulas.  Records are left
# out only by a computed condition criterion: where the reference's OWN FP32
# arithmetic (the oracle's FP32 port, bit-identical to the reference build compiled
# on the host) already differs from FP64 by more than half the tolerance, the
# quantity is ill-conditioned in FP32 at that input -- e.g. the GGX D term near its
# peak at low roughness, where 1 - NoH^2 (1 - a^2) cancels and amplifies the
# rounding of NoH by ~1/a^2 -- and no FP32 evaluation of the same formula can be
# held to 1e-5 there.  The excluded fraction is capped per column below (measured
# on these seeded inputs; roughness U(0.05, 1)).
TOL = 1e-5
COND = 0.5 * TOL
BSDF_COLS = [c for c in range(34) if c not in (8, 16)]  # 8, 16: integer outputs
# per-column cap on the excluded fraction: the VNDF sample pdf (7) is the D term at
# the sampled half-vector, ill-conditioned for roughness below ~0.3
EXCLUDE_CAP = {7: 0.30}
EXCLUDE_CAP_DEFAULT = 0.02


def _rel(x, r):
    with np.errstate(divide="ignore", invalid="ignore"):
        d = np.abs(x - r) / np.abs(r)
    d[(r == 0) & (x == 0)] = 0.0
    d[(r == 0) & (x != 0)] = np.inf
    return d


def check_against_fp64(g, o32, o64, label):
    """Max relative error of g vs o64 over the well-conditioned finite records of
    every column; returns {column: (max error, excluded fraction)}."""
    report = {}
    for c in BSDF_COLS:
        fin = np.isfinite(o64[:, c]) & np.isfinite(o32[:, c])
        # non-finite where the reference's FP32 is non-finite (e.g. the 0/0 pdf of A14);
        # an ulp of sin / cos may move a record across that edge: at most 1 in 10^4
        assert (np.isfinite(g[:, c]) != np.isfinite(o32[:, c])).mean() <= 1e-4, (label, c)
        fin &= np.isfinite(g[:, c])
        cond = fin & (_rel(o32[:, c], o64[:, c]) <= COND)
        excluded = 1.0 - cond.sum() / max(1, fin.sum())
        assert excluded <= EXCLUDE_CAP.get(c, EXCLUDE_CAP_DEFAULT), (label, c, excluded)
        err = float(_rel(g[cond, c], o64[cond, c]).max()) if cond.any() else 0.0
        report[c] = (err, excluded)
        assert err < TOL, (label, c, err, excluded)
    return report
