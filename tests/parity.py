"""Parity metrics between a GPU result and the FP64 oracle (test helper).

Acceptance (the tracking bar): on the points where the oracle reports a
match, offsets within 0.01 px (complex matches) / 0.02 px (amplitude
matches) on at least 99.5 % of them, and identical match types on at least
99.5 % of all points (differences only at threshold ties).
"""
import numpy as np

TOL_CMPX = 0.01
TOL_AMP = 0.02


def compare_track(gpu, orc, min_frac=0.995):
    t_g, t_o = gpu["type"], orc["type"]
    matched = t_o > 0
    same_type = float((t_g == t_o).mean())
    both = matched & (t_g > 0)
    tol = np.where(t_o == 1, TOL_CMPX, TOL_AMP)
    dr = np.abs(gpu["offR"].astype(np.float64) - orc["offR"])
    da = np.abs(gpu["offA"].astype(np.float64) - orc["offA"])
    ok = both & (dr <= tol) & (da <= tol)
    n_match = int(matched.sum())
    frac_ok = float(ok.sum()) / max(1, n_match)
    # failure encodings must agree exactly where neither matched
    neither = (~matched) & (t_g == 0)
    fail_enc = bool((gpu["offR"][neither] == orc["offR"][neither]).all())
    corr_rel = np.abs(gpu["corr"].astype(np.float64) - orc["corr"]) / np.maximum(1e-6, np.abs(orc["corr"]))
    stats = {
        "n_points": int(t_o.size),
        "n_match_oracle": n_match,
        "n_match_gpu": int((t_g > 0).sum()),
        "frac_offsets_ok": frac_ok,
        "frac_same_type": same_type,
        "fail_encoding_equal": fail_enc,
        "corr_rel_p99": float(np.percentile(corr_rel[both], 99)) if both.any() else 0.0,
        "max_off_err_px": float(np.max(np.maximum(dr, da)[both])) if both.any() else 0.0,
        "median_off_err_px": float(np.median(np.maximum(dr, da)[both])) if both.any() else 0.0,
    }
    stats["pass"] = frac_ok >= min_frac and same_type >= min_frac and fail_enc
    return stats
