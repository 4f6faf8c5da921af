"""CPU oracle of the overlap report -- TEST INFRASTRUCTURE ONLY.

Restates the pair-overlap diagnostic of the reference's analysis package
(rcptools/overlap.py:7-113, overlap_report) by brute force over all pairs:
candidates are the pairs i < j whose minimum-image distance is at most
2 * max(D)/2 (the reference's KD-tree query radius, overlap.py:53), the
displacement is pos[i] - pos[j] with the image removed by round-half-even
(overlap.py:63-65), and a candidate overlaps when (r_i + r_j) - |d| > 0.
Fractions: overlap / (r_i + r_j) ("sum", the convergence gate's convention)
and overlap / min(r_i, r_j) ("min"). Pinned by tests/test_overlap_oracle.py
against tests/golden/overlap_report.npz (the reference function's own output
on the golden packings).
"""

from __future__ import annotations

import numpy as np


def overlap_pairs(pos, D, box=None, chunk=512):
    """Returns (pairs [m x 2] sorted by (i, j), frac_sum, frac_min,
    n_candidate_pairs)."""
    pos = np.asarray(pos, dtype=np.float64)
    D = np.asarray(D, dtype=np.float64)
    N = pos.shape[0]
    R = D / 2.0
    rq = 2.0 * R.max() if N else 0.0
    L = None if box is None else np.asarray(box, dtype=np.float64)
    pairs, fs, fm = [], [], []
    ncand = 0
    for i0 in range(0, N, chunk):
        i1 = min(N, i0 + chunk)
        delta = pos[i0:i1, None, :] - pos[None, :, :]
        with np.errstate(divide="ignore", invalid="ignore"):  # a zero box side gives NaN, as in the reference
            if L is not None:
                delta = delta - np.round(delta / L) * L
            dist = np.sqrt(np.sum(delta * delta, axis=2))
        ii, jj = np.meshgrid(np.arange(i0, i1), np.arange(N), indexing="ij")
        upper = jj > ii
        cand = upper & (dist <= rq)
        ncand += int(cand.sum())
        rsum = R[ii] + R[jj]
        ov = rsum - dist
        hit = cand & (ov > 0)
        a, b = np.nonzero(hit)
        pi, pj = ii[a, b], jj[a, b]
        o = ov[a, b]
        pairs.append(np.stack([pi, pj], axis=1))
        fs.append(o / rsum[a, b])
        fm.append(o / np.minimum(R[pi], R[pj]))
    if not pairs:
        return np.zeros((0, 2), np.int64), np.zeros(0), np.zeros(0), 0
    P = np.concatenate(pairs).astype(np.int64)
    S = np.concatenate(fs)
    M = np.concatenate(fm)
    order = np.lexsort((P[:, 1], P[:, 0]))
    return P[order], S[order], M[order], ncand
