"""Error measures of the parity tests (shared by tests, smoke() and bench.py).

* acceleration error of a stage: max_i |a_i - a_i'| / sum_{j!=i} |GM_j / r_ij^2|, with
  a_i = gaccel + daccel + naccel; the magnitude sum keeps the measure finite for bodies whose
  forces cancel.
* position error: max_i |r_i - r_i'| / |r_i - r_0| (body 0 is the central star).
"""
import numpy as np

R_HI, R_LO, GM = 0, 3, 39
NACC, DACC, GACC = 67, 70, 76
DTQ = 73


def positions(pl):
    return pl[R_HI:R_HI + 3] + pl[R_LO:R_LO + 3]


def total_acc(pl):
    return (pl[GACC:GACC + 3] + pl[DACC:DACC + 3]) + pl[NACC:NACC + 3]


def newton_scale(pl):
    """sum_j GM_j / |r_ij|^2 for every body i."""
    r = positions(pl).T
    gm = pl[GM]
    d = r[None, :, :] - r[:, None, :]
    r2 = (d * d).sum(-1)
    np.fill_diagonal(r2, np.inf)
    return (gm[None, :] / r2).sum(1)


def accel_error(pl_a, pl_b, ref_pl=None):
    ref_pl = pl_b if ref_pl is None else ref_pl
    da = np.abs(total_acc(pl_a) - total_acc(pl_b)).max(0)
    return float((da / newton_scale(ref_pl)).max())


def position_error(pl_a, pl_b):
    ra, rb = positions(pl_a), positions(pl_b)
    dr = np.sqrt(((pl_a[R_HI:R_HI + 3] - pl_b[R_HI:R_HI + 3]) + (pl_a[R_LO:R_LO + 3] - pl_b[R_LO:R_LO + 3])) ** 2).sum(0)
    dist = np.sqrt(((rb - rb[:, :1]) ** 2).sum(0))
    dist[0] = np.sqrt((rb[:, 0] ** 2).sum()) or 1.0
    return float((dr / dist).max())


def rel_err(a, b, floor=0.0):
    a, b = np.asarray(a), np.asarray(b)
    return float((np.abs(a - b) / np.maximum(np.abs(b), floor)).max())
