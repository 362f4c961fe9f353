"""Certificate checks for the tests: the reference's own checkers (src/core/certificate.cpp)
through the reference build when it is present, else a numpy restatement of the same rules
(pinned against the reference build by tests/test_certificates_cpu.py)."""
import numpy as np

import oracle


def _fin(v):
    return np.abs(v) < 1e30


def farkas_numpy(lp, y):
    """farkas_proves_infeasible (src/core/certificate.cpp:29-119)."""
    y = np.asarray(y, dtype=np.float64)
    if not np.any(y != 0):
        return False, "every multiplier is zero"
    if np.any((y > 0) & ~_fin(lp.row_lower)) or np.any((y < 0) & ~_fin(lp.row_upper)):
        return False, "a multiplier leans on a missing row bound"
    required = float(np.sum(np.where(y > 0, y * np.where(_fin(lp.row_lower), lp.row_lower, 0.0),
                                     np.where(y < 0, y * np.where(_fin(lp.row_upper),
                                                                  lp.row_upper, 0.0), 0.0))))
    a = lp.to_scipy_csc()
    d = a.T @ y
    terms = abs(a.multiply(y[:, None])) if lp.num_nonzeros else None
    scale = float(terms.max()) if terms is not None else 0.0
    thr = 1e-11 * max(1.0, scale)
    up, dn = d > thr, d < -thr
    if np.any(up & ~_fin(lp.col_upper)) or np.any(dn & ~_fin(lp.col_lower)):
        return False, "the aggregate leans on a free column"
    reach = float(np.sum(np.where(up, d * np.where(_fin(lp.col_upper), lp.col_upper, 0.0), 0.0)
                         + np.where(dn, d * np.where(_fin(lp.col_lower), lp.col_lower, 0.0), 0.0)))
    margin = required - reach
    return margin > 1e-7 * max(1.0, abs(required), abs(reach), scale), f"margin {margin}"


def ray_numpy(lp, d):
    """ray_proves_unbounded (src/core/certificate.cpp:121-218) for an LP."""
    d = np.asarray(d, dtype=np.float64)
    mag = float(np.max(np.abs(d))) if d.size else 0.0
    if mag == 0.0:
        return False, "zero direction"
    moving = 1e-7 * mag
    if np.any((d > moving) & _fin(lp.col_upper)) or np.any((d < -moving) & _fin(lp.col_lower)):
        return False, "moves a column against its bound"
    a = lp.to_scipy_csc()
    act = a @ d
    scale = float(abs(a.multiply(d[None, :])).max()) if lp.num_nonzeros else 0.0
    rm = 1e-7 * max(1.0, scale)
    if np.any((act > rm) & _fin(lp.row_upper)) or np.any((act < -rm) & _fin(lp.row_lower)):
        return False, "moves a row against its bound"
    sense = -1.0 if lp.maximize else 1.0
    terms = sense * lp.cost * d
    imp = float(np.sum(terms))
    return imp < -1e-7 * max(1.0, float(np.max(np.abs(terms)))), f"improvement {imp}"


def farkas_ok(lp, y):
    if oracle.ref_available():
        return oracle.ref_farkas_check(lp, y)
    return farkas_numpy(lp, y)


def ray_ok(lp, d):
    if oracle.ref_available():
        return oracle.ref_ray_check(lp, d)
    return ray_numpy(lp, d)
