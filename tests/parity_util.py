"""Shared checks of the parity tests: how a ray result of the engine is
compared with the reference pipeline (the reference's own SoftwareBVH tree
traversed by the restated software_bvh_bvh4.comp).

In the shader's arithmetic (the engine's Moller-Trumbore mode) the two may
differ only where two triangles that share a vertex are hit at the same t
and the trees visit them in different orders (edge ties); those rays are
counted and must stay under 1e-5 of the rays, and t agrees within 1e-6
relative.  With the engine's default watertight test the triangle test
itself differs: the shader's test culls triangles nearly parallel to the ray
(|a| = |e1 . (d x e2)| < 1e-7, software_bvh_bvh4.comp:170), leaves cracks at
shared edges, and loses the barycentrics to cancellation when the origin is
far from a small triangle.  There, every disagreement must be reproduced by
tracing the same ray with the engine in the shader's arithmetic on the same
tree (the difference lies in the triangle test alone); such rays are counted
by kind."""
import numpy as np

GRAZE_BARY = 1e-5
GRAZE_FRACTION = 1e-5
MT_EPS = np.float32(1e-7)
T_REL = 1e-6


def mt_determinant(ray, v):
    """The shader's Moller-Trumbore determinant a = e1 . (d x e2) in float32
    (software_bvh_bvh4.comp:166-170)."""
    d = np.asarray(ray[4:7], np.float32)
    e1 = (v[1] - v[0]).astype(np.float32)
    e2 = (v[2] - v[0]).astype(np.float32)
    h = np.array([d[1] * e2[2] - d[2] * e2[1], d[2] * e2[0] - d[0] * e2[2], d[0] * e2[1] - d[1] * e2[0]],
                 np.float32)
    return np.float32(np.float32(e1[0] * h[0] + e1[1] * h[1]) + e1[2] * h[2])


def edge_distance(ray, v):
    """Smallest barycentric coordinate (float64) of the ray's crossing of the
    triangle's plane: ~0 means the ray passes along an edge.  ray: float32[8]
    (origin, tmin, direction, tmax); v: float32[3, 3] vertices."""
    o, d = np.asarray(ray[0:3], np.float64), np.asarray(ray[4:7], np.float64)
    v = v.astype(np.float64)
    e1, e2 = v[1] - v[0], v[2] - v[0]
    n = np.cross(e1, e2)
    t = np.dot(v[0] - o, n) / np.dot(d, n)
    p = o + t * d
    area = np.dot(n, n)
    b1 = np.dot(np.cross(p - v[0], e2), -n) / area
    b2 = np.dot(np.cross(e1, p - v[0]), n) / area
    return min(abs(1 - b1 - b2), abs(b1), abs(b2))


def ray_rows(rays):
    """rays as float32 [n, 8] whatever their dtype (structured or plain)."""
    r = np.ascontiguousarray(rays)
    return r.view(np.float32).reshape(-1, 8)


def graze_report(pos, idx, rays, ours_hit, ours_prim, ref_hit, ref_prim, closest=True, ours_t=None, ref_t=None,
                 mt_hit=None, mt_prim=None):
    """Disagreements between the engine and the reference pipeline, sorted
    into explained kinds, and the rays no kind explains.

    A ray is compared on hit/miss and, for closest-hit rays, on the
    primitive (original ids; where one side hits and the other misses, the
    hit side's primitive must be given; for any-hit rays ours_prim may come
    from a closest-hit trace of those rays).  Kinds:
      "edge"     the triangle one side hit and the other passed lies within
                 1e-5 (barycentric) of an edge of the ray's crossing, or both
                 hit triangles share a vertex at equal t (a tie on the edge);
      "parallel" the engine hit a triangle, no farther than the reference's
                 hit, that the shader's Moller-Trumbore test culls as parallel
                 to the ray (|a| < 1e-7, software_bvh_bvh4.comp:170);
      "test"     (mt_hit given: the engine's results for the same rays in the
                 shader's arithmetic on the same tree) none of the above, but
                 the engine in the shader's arithmetic gives the reference's
                 result: the difference lies in the triangle test.
    Returns (indices of all disagreements, dict kind -> count, unexplained)."""
    pos = np.asarray(pos, np.float32).reshape(-1, 3)
    tri = np.asarray(idx, np.uint32).reshape(-1, 3)
    rr = ray_rows(rays)
    ours_hit = np.asarray(ours_hit).astype(np.uint32)
    ref_hit = np.asarray(ref_hit).astype(np.uint32)
    differ = ours_hit != ref_hit
    if closest:
        differ |= (ours_hit == 1) & (ref_hit == 1) & (ours_prim != ref_prim)
    dis = np.nonzero(differ)[0]
    kinds = {"edge": 0, "parallel": 0, "test": 0}
    unexplained = []

    def grazes(i, pid):
        return edge_distance(rr[i], pos[tri[pid]]) <= GRAZE_BARY

    def culled(i, pid):
        return abs(mt_determinant(rr[i], pos[tri[pid]])) < MT_EPS

    for i in dis:
        kind = None
        if ours_hit[i] != ref_hit[i]:
            pid = ours_prim[i] if ours_hit[i] else ref_prim[i]
            if grazes(i, pid):
                kind = "edge"
            elif ours_hit[i] and culled(i, pid):
                kind = "parallel"
        else:
            a, b = int(ours_prim[i]), int(ref_prim[i])
            to = None if ours_t is None else np.float64(ours_t[i])
            tr_ = None if ref_t is None else np.float64(ref_t[i])
            shared = bool(set(tri[a].tolist()) & set(tri[b].tolist()))
            if shared and (to is None or abs(to - tr_) <= T_REL * abs(tr_)):
                kind = "edge"
            elif to is not None and to <= tr_ and (culled(i, a) or grazes(i, a)):
                kind = "parallel" if culled(i, a) else "edge"
            elif to is not None and tr_ < to and grazes(i, b):
                kind = "edge"
        if kind is None and mt_hit is not None:
            same_flag = int(mt_hit[i]) == int(ref_hit[i])
            if same_flag and (not closest or ref_hit[i] == 0 or int(mt_prim[i]) == int(ref_prim[i])):
                kind = "test"
        if kind is None:
            unexplained.append(int(i))
        else:
            kinds[kind] += 1
    return dis, kinds, unexplained


def assert_t_close(ours_t, ref_t, mask, mt_t=None):
    """Hit distances of rays both pipelines hit on the same primitive agree
    within 1e-6 relative; with mt_t (the engine's t in the shader's
    arithmetic), a ray off by more must have mt_t equal to the reference's t
    (the two triangle tests round t differently on rays that graze the
    triangle's plane).  Returns the number of such rays."""
    if not mask.any():
        return 0
    rel = np.abs(ours_t.astype(np.float64) - ref_t) / np.abs(ref_t.astype(np.float64))
    off = mask & (rel > T_REL)
    if mt_t is None:
        assert not off.any(), rel[mask].max()
        return 0
    assert np.array_equal(np.asarray(mt_t)[off].view(np.uint32), np.asarray(ref_t)[off].view(np.uint32)), \
        rel[off].max()
    return int(off.sum())
