"""Helpers for the hit-id agreement checks (parity rule 4): a disagreement
between two intersection forms on the same tree is explained when both hit
with equal t (a tie between triangles sharing an edge or lying on top of each
other) or when one of the two hits lies within a relative 1e-5 of an edge of
its triangle (float64 barycentric coordinates), where the forms' last-ulp
differences decide inside / outside."""
import numpy as np


def bary_margin(verts, tri, ray):
    """Smallest barycentric coordinate (float64) of the ray's hit with the
    triangle's plane, or None for a ray parallel to it."""
    p1, p2, p3 = (verts[tri[k], :3].astype(np.float64) for k in range(3))
    o, d = ray[:3].astype(np.float64), ray[4:7].astype(np.float64)
    e1, e2 = p2 - p1, p3 - p1
    h = np.cross(d, e2)
    a = e1 @ h
    if abs(a) < 1e-300:
        return None
    f = 1.0 / a
    s = o - p1
    u = f * (s @ h)
    w = f * (d @ np.cross(s, e1))
    return min(u, w, 1.0 - u - w)


def explain(verts, tris, rays, ids_a, t_a, ids_b, t_b, tol=1e-5):
    """(number of disagreeing rays, number of them explained)."""
    dis = np.nonzero(ids_a != ids_b)[0]
    ok = 0
    for i in dis:
        a, b = int(ids_a[i]), int(ids_b[i])
        if a >= 0 and b >= 0 and abs(float(t_a[i]) - float(t_b[i])) <= tol * max(abs(float(t_a[i])), 1e-30):
            ok += 1
            continue
        m = [bary_margin(verts, tris[k], rays[i]) for k in (a, b) if k >= 0]
        m = [abs(x) for x in m if x is not None]
        if m and min(m) <= tol:
            ok += 1
    return len(dis), ok
