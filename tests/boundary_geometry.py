"""Seeded boundary-tier inputs for the tests: a disk (or cylinder through all z
layers) of radius R centred on the grid.

The planner that computes these arrays from a geometry is outside the
time-stepper; any arrays of this shape are valid inputs to the tiers.  This
generator gives plausible ones:
  - volume fraction phi: share of sub x sub sample points of the cell inside;
  - face links: share of sub sample points of each x/y face inside (z faces = phi);
  - distances: from the cell centre to the boundary along each in-plane axis
    (bisection), the cell size when the neighbour centre is inside, 0 when the
    centre is outside; the cell size along z;
  - sparse demag correction: targets = partial cells (0 < phi < 1), sources =
    their 3 x 3 in-plane neighbourhood (-1 outside the grid or the body), random
    symmetric tensors of size ~1e-3 (xx, xy, xz, yy, yz, zz).
"""
import numpy as np


def disk_geometry(nx, ny, nz, dx, dy, dz, radius, sub=4, seed=5):
    xc = (np.arange(nx) + 0.5) * dx - nx * dx / 2
    yc = (np.arange(ny) + 0.5) * dy - ny * dy / 2
    X, Y = np.meshgrid(xc, yc)              # [ny, nx]
    off = (np.arange(sub) + 0.5) / sub - 0.5
    inside = lambda x, y: x * x + y * y <= radius * radius

    phi = np.zeros((ny, nx))
    for a in off:
        for b in off:
            phi += inside(X + a * dx, Y + b * dy)
    phi /= sub * sub

    def face(px, py, along_x):
        acc = np.zeros((ny, nx))
        for a in off:
            acc += inside(px + (0 if along_x else a * dx), py + (a * dy if along_x else 0))
        return acc / sub

    fxp = face(X + dx / 2, Y, True)
    fxm = face(X - dx / 2, Y, True)
    fyp = face(X, Y + dy / 2, False)
    fym = face(X, Y - dy / 2, False)

    def dist(ux, uy, d):
        out = np.zeros((ny, nx))
        cin = inside(X, Y)
        far = inside(X + ux * d, Y + uy * d)
        out[cin & far] = d
        lo = np.zeros((ny, nx))
        hi = np.full((ny, nx), d)
        for _ in range(40):
            mid = 0.5 * (lo + hi)
            ok = inside(X + ux * mid, Y + uy * mid)
            lo = np.where(ok, mid, lo)
            hi = np.where(ok, hi, mid)
        sel = cin & ~far
        out[sel] = lo[sel]
        return out

    dxp, dxm = dist(1, 0, dx), dist(-1, 0, dx)
    dyp, dym = dist(0, 1, dy), dist(0, -1, dy)

    rep = lambda a: np.repeat(a[None], nz, axis=0).reshape(-1)
    vf = rep(phi)
    faces = [rep(fxp), rep(fxm), rep(fyp), rep(fym), rep(phi), rep(phi)]
    deltas = [rep(dxp), rep(dxm), rep(dyp), rep(dym), np.full(vf.size, dz), np.full(vf.size, dz)]
    mask = (vf > 0).astype(np.uint8)

    rng = np.random.default_rng(seed)
    targets, sources, tensors = [], [], []
    for z in range(nz):
        for y in range(ny):
            for x in range(nx):
                i = (z * ny + y) * nx + x
                if not (0.0 < vf[i] < 1.0):
                    continue
                targets.append(i)
                row = []
                for oy in (-1, 0, 1):
                    for ox in (-1, 0, 1):
                        xx, yy = x + ox, y + oy
                        j = (z * ny + yy) * nx + xx
                        ok = 0 <= xx < nx and 0 <= yy < ny and vf[j] > 0
                        row.append(j if ok else -1)
                sources.append(row)
                tensors.append(rng.uniform(-1e-3, 1e-3, size=(9, 6)))
    corr = (np.array(targets, dtype=np.int32), np.array(sources, dtype=np.int32),
            np.array(tensors, dtype=np.float64))
    return dict(vf=vf, faces=faces, deltas=deltas, mask=mask, corr=corr)
