"""Hit-parity bookkeeping shared by the GPU ray tests.

A GPU hit agrees with the oracle/reference when the primitive id (and plane
flag) is identical and t matches within 1e-5 relative. Where two surfaces are
hit at the same distance (coplanar faces such as a box's bottom lying on the
floor, or a ray through a shared edge) the id is decided by rounding: the
reference's own BVH and brute force disagree there. Such a ray counts as a tie
when both report a hit and the GPU's t matches the oracle's within 1e-5.
"""
import numpy as np

T_REL = 1e-5


def hit_parity(g_t, g_prim, g_plane, r_t, r_prim, r_plane, t_rel=T_REL):
    g_prim = np.asarray(g_prim)
    r_prim = np.asarray(r_prim)
    g_hit = g_prim >= 0
    r_hit = r_prim >= 0
    same_id = (g_prim == r_prim) & (np.asarray(g_plane) == np.asarray(r_plane))
    t_close = np.abs(np.asarray(g_t, np.float64) - np.asarray(r_t, np.float64)) <= t_rel * np.abs(r_t)
    strict = same_id & ((~r_hit) | t_close)
    tie = (~same_id) & g_hit & r_hit & t_close
    return {
        "n": int(len(g_prim)),
        "strict": float(strict.mean()),
        "accepted": float((strict | tie).mean()),
        "ties": int(tie.sum()),
        "fail_idx": np.nonzero(~(strict | tie))[0],
        "hit_rate": float(r_hit.mean()),
    }


def t_share(g_t, g_prim, r_t, r_prim, t_rel=T_REL):
    """Share of the rays both sides hit whose GPU t is within t_rel of the reference's."""
    both = (np.asarray(g_prim) >= 0) & (np.asarray(r_prim) >= 0)
    g = np.asarray(g_t, np.float64)[both]
    r = np.asarray(r_t, np.float64)[both]
    return float(np.mean(np.abs(g - r) <= t_rel * np.abs(r))) if both.any() else 1.0
