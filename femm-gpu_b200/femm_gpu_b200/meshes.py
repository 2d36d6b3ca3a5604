"""Seeded synthetic meshes for the benchmark workloads.

Each generator is deterministic in its arguments.  The workloads are:

* ``square_linear(m)`` -- plain linear planar solve: 0.1 m square, m x m quads split
  along the lower-left -> upper-right diagonal, a centred 0.04 m iron block with
  mu_r = 1000, two 0.01 x 0.03 m coil slabs driven at J = +/-1e6 A/m^2 by one
  series circuit at 10 A, air elsewhere, A = 0 on the outer boundary.  m = 64 gives
  4,225 nodes / 8,192 triangles.
* ``square_nonlinear(m, seed)`` -- the same layout with interior nodes jittered by
  U(+/-0.3 h), the iron on a 24-point B-H table sampled from B = 2 H / (200 + H)
  (H = 0 and 23 log-spaced points in [10, 2e5] A/m), a 0.005 m NdFe-like magnet
  strip (mu_r = 1.05, Hc = 9e5 A/m, seeded angle) and three series circuits.
  m = 500 gives 251,001 nodes / 500,000 triangles; m = 1414 gives 2,002,225 nodes.
* ``axisymmetric_plunger(mr, mz)`` -- r-z solenoid plunger: r in [0, 0.05],
  z in [-0.05, 0.05], iron plunger r < 0.01 on the same B-H table, two coils in
  r in [0.015, 0.025], A = 0 on the axis and outer boundary.

Jittered meshes can invert a few triangles (about 10 in 500,000 at 0.3 h).  The
generator repairs them deterministically: nodes of any triangle whose area falls
below 5 % of the undistorted area get their jitter halved, repeatedly, until every
triangle is well shaped.
"""
from __future__ import annotations

import numpy as np

from .model import AXISYMMETRIC, MU0, PLANAR, AirGap, Model

SIDE_M = 0.1


def bh_table_saturating(points: int = 24):
    """B = 2 H / (200 + H): H = 0 plus (points - 1) log-spaced values in [10, 2e5] A/m."""
    h = np.concatenate([[0.0], np.logspace(1.0, np.log10(2.0e5), points - 1)])
    b = 2.0 * h / (200.0 + h)
    return b, h


def _structured(m: int, width: float, height: float, x0: float = 0.0, y0: float = 0.0):
    nx, ny = m if isinstance(m, tuple) else (m, m)
    xs = x0 + np.linspace(0.0, width, nx + 1)
    ys = y0 + np.linspace(0.0, height, ny + 1)
    X, Y = np.meshgrid(xs, ys)  # row = y, column = x -> node = j * (nx + 1) + i
    xy = np.stack([X.ravel(), Y.ravel()], axis=1)
    j, i = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    ll = (j * (nx + 1) + i).ravel()
    lr = ll + 1
    ul = ll + (nx + 1)
    ur = ul + 1
    tri = np.empty((2 * ll.size, 3), dtype=np.int64)
    tri[0::2] = np.stack([ll, lr, ur], axis=1)
    tri[1::2] = np.stack([ll, ur, ul], axis=1)
    return xy, tri.astype(np.int32), nx, ny


def _signed_area2(xy, tri):
    p0, p1, p2 = xy[tri[:, 0]], xy[tri[:, 1]], xy[tri[:, 2]]
    return (p1[:, 0] - p0[:, 0]) * (p2[:, 1] - p0[:, 1]) - (p2[:, 0] - p0[:, 0]) * (p1[:, 1] - p0[:, 1])


def _jitter(xy, tri, nx, ny, hx, hy, seed, fraction=0.3):
    rng = np.random.default_rng(seed)
    jit = rng.uniform(-fraction, fraction, size=xy.shape) * np.array([hx, hy])
    idx = np.arange(xy.shape[0])
    i = idx % (nx + 1)
    j = idx // (nx + 1)
    interior = (i > 0) & (i < nx) & (j > 0) & (j < ny)
    jit[~interior] = 0.0
    base = _signed_area2(xy, tri)
    for _ in range(64):
        moved = xy + jit
        area = _signed_area2(moved, tri)
        bad = area < 0.05 * base
        if not bad.any():
            return moved
        nodes = np.unique(tri[bad].ravel())
        jit[nodes] *= 0.5
    raise RuntimeError("jitter repair did not converge")


def _centroids(xy, tri):
    return xy[tri].mean(axis=1)


def _in_box(c, x0, x1, y0, y1):
    return (c[:, 0] >= x0) & (c[:, 0] <= x1) & (c[:, 1] >= y0) & (c[:, 1] <= y1)


def _boundary_nodes(nx, ny):
    idx = np.arange((nx + 1) * (ny + 1))
    i = idx % (nx + 1)
    j = idx // (nx + 1)
    return idx[(i == 0) | (i == nx) | (j == 0) | (j == ny)].astype(np.int32)


def square_linear(m: int = 64, current_a: float = 10.0) -> Model:
    """Linear planar workload; the circuit current is ``current_a`` (J = +/-1e6 at 10 A)."""
    xy, tri, nx, ny = _structured(m, SIDE_M, SIDE_M)
    c = _centroids(xy, tri)
    mat = np.zeros(tri.shape[0], np.int32)  # 0 air
    mat[_in_box(c, 0.03, 0.07, 0.03, 0.07)] = 1  # iron
    mat[_in_box(c, 0.015, 0.025, 0.035, 0.065)] = 2  # coil +
    mat[_in_box(c, 0.075, 0.085, 0.035, 0.065)] = 3  # coil -
    jpa = 1.0e6 / current_a
    nu_air = 1.0 / MU0
    return Model(
        xy=xy, tri=tri, tri_mat=mat,
        nu0=[nu_air, nu_air / 1000.0, nu_air, nu_air],
        alpha=[0.0, 0.0, 0.0, 0.0],
        j_per_a=[0.0, 0.0, jpa, -jpa],
        hc=[0.0, 0.0, 0.0, 0.0],
        mag_deg=[0.0, 0.0, 0.0, 0.0],
        curve_index=[-1, -1, -1, -1],
        circuit_index=[-1, -1, 0, 0],
        group=[0, 1, 2, 3],
        curves=[],
        dir_nodes=_boundary_nodes(nx, ny),
        dir_values=np.zeros(_boundary_nodes(nx, ny).size),
        circuit_count=1,
        depth_m=1.0,
        problem_type=PLANAR,
        name=f"square_linear_m{m}",
    )


def square_nonlinear(m: int = 500, seed: int = 2, magnet_deg: float | None = None,
                     jitter: float = 0.3) -> Model:
    """Nonlinear planar workload (iron B-H, PM strip, three series circuits)."""
    xy, tri, nx, ny = _structured(m, SIDE_M, SIDE_M)
    h = SIDE_M / m
    rng = np.random.default_rng(seed)
    if jitter > 0.0:
        xy = _jitter(xy, tri, nx, ny, h, h, seed, jitter)
    if magnet_deg is None:
        magnet_deg = float(rng.uniform(0.0, 360.0))
    c = _centroids(xy, tri)
    mat = np.zeros(tri.shape[0], np.int32)  # 0 air
    mat[_in_box(c, 0.03, 0.07, 0.03, 0.07)] = 1  # iron (B-H)
    mat[_in_box(c, 0.03, 0.07, 0.0175, 0.0225)] = 2  # magnet strip, 5 mm
    mat[_in_box(c, 0.015, 0.025, 0.035, 0.065)] = 3  # circuit 0
    mat[_in_box(c, 0.075, 0.085, 0.035, 0.065)] = 4  # circuit 1
    mat[_in_box(c, 0.035, 0.065, 0.075, 0.085)] = 5  # circuit 2
    nu_air = 1.0 / MU0
    jpa = 1.0e6 / 20.0  # 1e6 A/m^2 at the 20 A extreme of the current range
    b, hh = bh_table_saturating(24)
    bnd = _boundary_nodes(nx, ny)
    return Model(
        xy=xy, tri=tri, tri_mat=mat,
        nu0=[nu_air, nu_air / 1000.0, nu_air / 1.05, nu_air, nu_air, nu_air],
        alpha=np.zeros(6),
        j_per_a=[0.0, 0.0, 0.0, jpa, jpa, jpa],
        hc=[0.0, 0.0, 9.0e5, 0.0, 0.0, 0.0],
        mag_deg=[0.0, 0.0, magnet_deg, 0.0, 0.0, 0.0],
        curve_index=[-1, 0, -1, -1, -1, -1],
        circuit_index=[-1, -1, -1, 0, 1, 2],
        group=[0, 1, 2, 3, 4, 5],
        curves=[(b, hh)],
        dir_nodes=bnd,
        dir_values=np.zeros(bnd.size),
        circuit_count=3,
        depth_m=1.0,
        problem_type=PLANAR,
        name=f"square_nonlinear_m{m}_s{seed}",
    )


def seeded_currents(items: int, circuits: int, limit: float, seed: int) -> np.ndarray:
    """Circuit currents uniform in [-limit, limit] A, shape [items, circuits]."""
    rng = np.random.default_rng(seed)
    return rng.uniform(-limit, limit, size=(items, circuits))


def axisymmetric_plunger(mr: int = 223, mz: int = 446) -> Model:
    """Axisymmetric solenoid plunger (r = x, z = y); about 100k nodes at the defaults."""
    xy, tri, nx, ny = _structured((mr, mz), 0.05, 0.1, 0.0, -0.05)
    c = _centroids(xy, tri)
    mat = np.zeros(tri.shape[0], np.int32)
    mat[c[:, 0] < 0.01] = 1  # plunger
    mat[_in_box(c, 0.015, 0.025, 0.005, 0.03)] = 2  # coil 0
    mat[_in_box(c, 0.015, 0.025, -0.03, -0.005)] = 3  # coil 1
    nu_air = 1.0 / MU0
    jpa = 1.0e6 / 30.0
    b, hh = bh_table_saturating(24)
    bnd = _boundary_nodes(nx, ny)
    return Model(
        xy=xy, tri=tri, tri_mat=mat,
        nu0=[nu_air, nu_air / 1000.0, nu_air, nu_air],
        alpha=np.zeros(4),
        j_per_a=[0.0, 0.0, jpa, jpa],
        hc=np.zeros(4),
        mag_deg=np.zeros(4),
        curve_index=[-1, 0, -1, -1],
        circuit_index=[-1, -1, 0, 1],
        group=[0, 1, 2, 3],
        curves=[(b, hh)],
        dir_nodes=bnd,
        dir_values=np.zeros(bnd.size),
        circuit_count=2,
        depth_m=1.0,
        problem_type=AXISYMMETRIC,
        name=f"axisymmetric_plunger_{mr}x{mz}",
    )


def periodic_strip(m: int = 16, antiperiodic: bool = False, current_a: float = 12.0) -> Model:
    """Square strip with periodic (or anti-periodic) left/right edges and A = 0 top/bottom."""
    xy, tri, nx, ny = _structured(m, 0.01, 0.01)
    c = _centroids(xy, tri)
    mat = np.zeros(tri.shape[0], np.int32)
    coil = _in_box(c, 0.003, 0.007, 0.003, 0.007)
    mat[coil] = 1
    area = 0.5 * _signed_area2(xy, tri)[coil].sum()
    idx = np.arange(xy.shape[0])
    i = idx % (nx + 1)
    j = idx // (nx + 1)
    bnd = idx[(j == 0) | (j == ny)].astype(np.int32)
    left = idx[(i == 0) & (j > 0) & (j < ny)]
    right = idx[(i == nx) & (j > 0) & (j < ny)]
    nu_air = 1.0 / MU0
    return Model(
        xy=xy, tri=tri, tri_mat=mat,
        nu0=[nu_air, nu_air], alpha=[0.0, 0.0], j_per_a=[0.0, 1.0 / area], hc=[0.0, 0.0],
        mag_deg=[0.0, 0.0], curve_index=[-1, -1], circuit_index=[-1, 0], group=[0, 1], curves=[],
        dir_nodes=bnd, dir_values=np.zeros(bnd.size),
        con_a=left, con_b=right,
        con_sign=np.full(left.size, -1 if antiperiodic else 1, np.int8),
        circuit_count=1, depth_m=0.01, problem_type=PLANAR,
        name=f"{'anti' if antiperiodic else ''}periodic_strip_m{m}",
    )


def annular_sector(nr: int = 160, nt: int = 250, hc: float = 9.0e5, turns: float = 20.0) -> Model:
    """Rotor-stator quarter machine: r in [0.02, 0.06] m, a 90-degree sector with
    anti-periodic edges (4 poles: one surface magnet per sector), 12 stator slots (3 per
    sector), a 1 mm air gap.  Radially: rotor iron [0.020, 0.043) on the saturating B-H
    table; a 2 mm surface magnet [0.043, 0.045) over the central 60 degrees of the pole
    (mu_r 1.05, Hc = ``hc``, magnetised along the pole axis at 45 degrees), air between
    magnets; air gap [0.045, 0.046); stator [0.046, 0.060] with three 15-degree slots
    [0.046, 0.050), open at the gap, centred at 15, 45 and 75 degrees, each a coil of
    ``turns`` turns of one series circuit (3 circuits), iron elsewhere.  The proportions
    keep the 10 mm stator yoke near the knee of the B-H curve (about 1.8 T); the tooth
    corners still reach 2 T, so Newton takes some 25-30 relaxed iterations.  A = 0 on the
    outer radius; the shaft radius is a natural boundary.  nr x nt quads split into
    triangles on the polar grid; nr = 160, nt = 250 gives 40,411 nodes / 80,000
    triangles."""
    r0, r1 = 0.02, 0.06
    rs = np.linspace(r0, r1, nr + 1)
    ts = np.linspace(0.0, 0.5 * np.pi, nt + 1)
    T, R = np.meshgrid(ts, rs)  # row = r index, column = theta index: node = i * (nt + 1) + j
    xy = np.stack([(R * np.cos(T)).ravel(), (R * np.sin(T)).ravel()], axis=1)
    i, j = np.meshgrid(np.arange(nr), np.arange(nt), indexing="ij")
    a = (i * (nt + 1) + j).ravel()  # (r_i, t_j)
    b = a + 1                        # (r_i, t_j+1)
    c = a + (nt + 1)                 # (r_i+1, t_j)
    d = c + 1                        # (r_i+1, t_j+1)
    tri = np.empty((2 * a.size, 3), dtype=np.int64)
    # (r, theta) -> (x, y) preserves orientation for r > 0: (a, c, d) and (a, d, b) are CCW.
    tri[0::2] = np.stack([a, c, d], axis=1)
    tri[1::2] = np.stack([a, d, b], axis=1)
    tri = tri.astype(np.int32)
    cen = xy[tri].mean(axis=1)
    rc = np.hypot(cen[:, 0], cen[:, 1])
    tc = np.degrees(np.arctan2(cen[:, 1], cen[:, 0]))
    mat = np.zeros(tri.shape[0], np.int32)  # 0 air
    mat[rc < 0.043] = 1  # rotor iron
    mat[(rc >= 0.043) & (rc < 0.045) & (np.abs(tc - 45.0) <= 30.0)] = 2  # magnet
    stator = rc >= 0.046
    mat[stator] = 3  # stator iron
    for k, centre in enumerate((15.0, 45.0, 75.0)):
        slot = stator & (rc < 0.050) & (np.abs(tc - centre) <= 7.5)
        mat[slot] = 4 + k
    area = 0.5 * _signed_area2(xy, tri)
    jpa = [turns / area[mat == 4 + k].sum() for k in range(3)]
    nu_air = 1.0 / MU0
    b_t, h = bh_table_saturating(24)
    idx = np.arange(xy.shape[0])
    ii, jj = idx // (nt + 1), idx % (nt + 1)
    outer = idx[ii == nr].astype(np.int32)
    left = idx[(jj == 0) & (ii < nr)]
    right = idx[(jj == nt) & (ii < nr)]
    return Model(
        xy=xy, tri=tri, tri_mat=mat,
        nu0=[nu_air, nu_air, nu_air / 1.05, nu_air, nu_air, nu_air, nu_air],
        alpha=np.zeros(7),
        j_per_a=[0.0, 0.0, 0.0, 0.0, jpa[0], jpa[1], jpa[2]],
        hc=[0.0, 0.0, hc, 0.0, 0.0, 0.0, 0.0],
        mag_deg=[0.0, 0.0, 45.0, 0.0, 0.0, 0.0, 0.0],
        curve_index=[-1, 0, -1, 0, -1, -1, -1],
        circuit_index=[-1, -1, -1, -1, 0, 1, 2],
        group=[0, 1, 2, 3, 4, 5, 6],
        curves=[(b_t, h)],
        dir_nodes=outer,
        dir_values=np.zeros(outer.size),
        con_a=left, con_b=right,
        con_sign=np.full(left.size, -1, np.int8),
        circuit_count=3, depth_m=0.05, problem_type=PLANAR,
        name=f"annular_sector_{nr}x{nt}",
    )


def two_pole_machine(nr: int = 160, nt: int = 120, full: bool = False, hc: float = 9.0e5,
                     turns: float = 20.0) -> Model:
    """A two-pole surface-magnet machine, as the 180-degree sector [0, 180] degrees with
    antiperiodic edges (``full=False``) or the full 360-degree annulus (``full=True``, the
    sector and its 180-degree rotation, equal node numbering on the shared edges).

    r in [0.02, 0.06] m: rotor iron to 0.043 on the saturating B-H table, a 2 mm magnet
    [0.043, 0.045) over the central 120 degrees of the pole magnetised along +y (mu_r 1.05,
    Hc = ``hc``; the other pole's magnet points along +y too, an antiperiodic field), a 1 mm
    air gap, a stator with three 20-degree slots [0.046, 0.050) at 30, 90 and 150 degrees
    (circuits 0, 1, 2, ``turns`` turns each; the rotated copies in the full machine belong to
    the same circuits wound the other way).  Groups: air 50, rotor iron and magnets 20,
    stator 30, slots 40-42.  A = 0 on the outer radius."""
    r0, r1 = 0.02, 0.06
    span = 2.0 * np.pi if full else np.pi
    ntt = 2 * nt if full else nt
    rs = np.linspace(r0, r1, nr + 1)
    ts = np.linspace(0.0, span, ntt + 1)
    if full:
        ts = ts[:-1]  # the 360-degree seam closes on the first column
    cols = ts.size
    T, R = np.meshgrid(ts, rs)
    xy = np.stack([(R * np.cos(T)).ravel(), (R * np.sin(T)).ravel()], axis=1)
    if not full:
        xy[np.arange(nr + 1) * cols + (cols - 1), 1] = 0.0  # the 180-degree edge on y = 0 exactly
    else:
        # (-x, -y) partners exactly: the second half is the rotation of the first.
        half = nt
        for i in range(nr + 1):
            for j in range(half, cols):
                k, m = i * cols + j, i * cols + (j - half)
                xy[k] = -xy[m]
    i, j = np.meshgrid(np.arange(nr), np.arange(ntt), indexing="ij")
    jn = (j + 1) % cols if full else j + 1
    a = (i * cols + j).ravel()
    b = (i * cols + jn).ravel()
    c = ((i + 1) * cols + j).ravel()
    d = ((i + 1) * cols + jn).ravel()
    tri = np.empty((2 * a.size, 3), dtype=np.int64)
    tri[0::2] = np.stack([a, c, d], axis=1)
    tri[1::2] = np.stack([a, d, b], axis=1)
    tri = tri.astype(np.int32)
    cen = xy[tri].mean(axis=1)
    rc = np.hypot(cen[:, 0], cen[:, 1])
    tc = np.degrees(np.arctan2(cen[:, 1], cen[:, 0])) % 360.0
    upper = tc < 180.0
    tl = np.where(upper, tc, tc - 180.0)  # angle within its half
    mat = np.zeros(tri.shape[0], np.int32)  # 0 air
    mat[rc < 0.043] = 1
    mat[(rc >= 0.043) & (rc < 0.045) & (np.abs(tl - 90.0) <= 60.0)] = 2
    stator = rc >= 0.046
    mat[stator] = 3
    for k, centre in enumerate((30.0, 90.0, 150.0)):
        slot = stator & (rc < 0.050) & (np.abs(tl - centre) <= 10.0)
        mat[slot & upper] = 4 + k
        mat[slot & ~upper] = 7 + k
    area = 0.5 * _signed_area2(xy, tri)
    jpa = [turns / area[mat == 4 + k].sum() for k in range(3)]
    nu_air = 1.0 / MU0
    b_t, h = bh_table_saturating(24)
    idx = np.arange(xy.shape[0])
    ii, jj = idx // cols, idx % cols
    outer = idx[ii == nr].astype(np.int32)
    left = idx[(jj == 0) & (ii < nr)]
    right = idx[(jj == cols - 1) & (ii < nr)]
    M = 10 if full else 7  # the sector has no rotated slot copies
    return Model(
        xy=xy, tri=tri, tri_mat=mat,
        nu0=([nu_air, nu_air, nu_air / 1.05, nu_air] + [nu_air] * 6)[:M],
        alpha=np.zeros(M),
        j_per_a=([0.0, 0.0, 0.0, 0.0] + jpa + [-v for v in jpa])[:M],
        hc=([0.0, 0.0, hc] + [0.0] * 7)[:M],
        mag_deg=([0.0, 0.0, 90.0] + [0.0] * 7)[:M],
        curve_index=([-1, 0, -1, 0] + [-1] * 6)[:M],
        circuit_index=[-1, -1, -1, -1, 0, 1, 2, 0, 1, 2][:M],
        group=[50, 20, 20, 30, 40, 41, 42, 40, 41, 42][:M],
        curves=[(b_t, h)],
        dir_nodes=outer,
        dir_values=np.zeros(outer.size),
        con_a=np.zeros(0, np.int32) if full else left, con_b=np.zeros(0, np.int32) if full else right,
        con_sign=np.zeros(0, np.int8) if full else np.full(left.size, -1, np.int8),
        circuit_count=3, depth_m=0.05, problem_type=PLANAR,
        name=f"two_pole_{'full' if full else 'sector'}_{nr}x{nt}",
    )


def sliding_band_machine(nr: int = 160, nt: int = 120, rotor_deg: float = 0.0, hc: float = 9.0e5,
                         turns: float = 20.0, sector: bool = False) -> Model:
    """The two-pole machine of ``two_pole_machine`` with its 1 mm air gap [0.045, 0.046] m
    left untriangulated and spanned by one native air-gap element (FEMM's AGE).  The rotor
    (r <= 0.045: iron, magnets and the air between them) and the stator (r >= 0.046) are
    meshed separately on polar grids of the same radial step 0.04 / ``nr`` and ``nt``
    uniform columns per half turn; the rotor mesh, magnets included, is turned by
    ``rotor_deg``.  ``sector=False``: the full machine, a periodic band over 360 degrees.
    ``sector=True``: the half [0, 180] degrees with anti-periodic edges (the 180-degree
    nodes partner the 0-degree ones), the band over 180 degrees, anti-periodic, the three
    slots of the upper half only (materials 0-6).  The band's records follow FEMM's
    preprocessor: each ring's nodes and their copies around the full turn (copy signs -1
    for odd copies of an anti-periodic sector) sorted by angle in [0, 360), point p
    bracketed by ring entries p - 1 and p, each ring's shift = the angle of its first entry
    in units of one column.  Groups: air 50, rotor 20, stator 30, slots 40-42.  A = 0 on
    the outer radius."""
    h = 0.04 / nr
    rows_r, rows_s = int(round(0.025 / h)), int(round(0.014 / h))
    if abs(rows_r * h - 0.025) > 1e-12 or abs(rows_s * h - 0.014) > 1e-12:
        raise ValueError("nr must put the gap radii 0.045 and 0.046 m on grid rows")
    ring = nt if sector else 2 * nt           # ring nodes of the model (one per column)
    cols = nt + 1 if sector else 2 * nt       # mesh columns (the sector keeps its 180-degree edge)
    dt = 180.0 / nt
    rot = np.radians(rotor_deg)

    def polar(r_in, r_out, rows, turn):
        rs = np.linspace(r_in, r_out, rows + 1)
        ts = np.radians(np.arange(cols) * dt) + turn
        T, R = np.meshgrid(ts, rs)
        xy = np.stack([(R * np.cos(T)).ravel(), (R * np.sin(T)).ravel()], axis=1)
        if sector:  # the 180-degree edge is the exact half-turn of the 0-degree edge
            edge = np.arange(rows + 1) * cols
            xy[edge + cols - 1] = -xy[edge]
        i, j = np.meshgrid(np.arange(rows), np.arange(cols - 1 if sector else cols), indexing="ij")
        a = (i * cols + j).ravel()
        b = (i * cols + (j + 1) % cols).ravel()
        c = a + cols
        d = b + cols
        tri = np.empty((2 * a.size, 3), np.int64)
        tri[0::2] = np.stack([a, c, d], axis=1)
        tri[1::2] = np.stack([a, d, b], axis=1)
        return xy, tri

    xy_r, tri_r = polar(0.02, 0.045, rows_r, rot)
    xy_s, tri_s = polar(0.046, 0.06, rows_s, 0.0)
    off = xy_r.shape[0]
    xy = np.concatenate([xy_r, xy_s])
    tri = np.concatenate([tri_r, tri_s + off]).astype(np.int32)
    cen = xy[tri].mean(axis=1)
    rc = np.hypot(cen[:, 0], cen[:, 1])
    tc = np.degrees(np.arctan2(cen[:, 1], cen[:, 0]))
    rotor = np.arange(tri.shape[0]) < tri_r.shape[0]
    body = np.where(rotor, tc - rotor_deg, tc) % 360.0  # rotor parts move with the rotor
    upper = body < 180.0
    tl = np.where(upper, body, body - 180.0)
    mat = np.zeros(tri.shape[0], np.int32)
    mat[rotor & (rc < 0.043)] = 1
    mat[rotor & (rc >= 0.043) & (np.abs(tl - 90.0) <= 60.0)] = 2
    stator = ~rotor
    mat[stator] = 3
    for k, centre in enumerate((30.0, 90.0, 150.0)):
        slot = stator & (rc < 0.050) & (np.abs(tl - centre) <= 10.0)
        mat[slot & upper] = 4 + k
        mat[slot & ~upper] = 7 + k
    M = 7 if sector else 10
    area = 0.5 * _signed_area2(xy, tri)
    jpa = [turns / area[mat == 4 + k].sum() for k in range(3)]
    nu_air = 1.0 / MU0
    b_t, hh = bh_table_saturating(24)
    outer = (off + rows_s * cols + np.arange(cols)).astype(np.int32)
    con_a, con_b = np.zeros(0, np.int32), np.zeros(0, np.int32)
    if sector:  # 0-degree edge -> 180-degree edge, every row but the fixed outer one
        left = np.concatenate([np.arange(rows_r + 1) * cols, off + np.arange(rows_s) * cols])
        con_a, con_b = left.astype(np.int32), (left + cols - 1).astype(np.int32)

    def records(first, shift_deg):
        # the model's ring nodes and, for a sector, their half-turn copies (sign -1)
        node = np.concatenate([first + np.arange(ring)] * (2 if sector else 1))
        sign = np.concatenate([np.ones(ring), -np.ones(ring)]) if sector else np.ones(ring)
        ang = (np.arange(node.size) * dt + shift_deg) % 360.0
        order = np.argsort(ang, kind="stable")
        return node[order], sign[order], ang[order[0]] / dt

    n_in, s_in, inner_shift = records(rows_r * cols, rotor_deg)
    n_out, s_out, outer_shift = records(off, 0.0)
    total = n_in.size
    p = np.arange(ring + 1)
    p1, p0 = p % total, (p - 1) % total
    nodes = np.stack([n_in[p0], n_in[p1], n_out[p0], n_out[p1]], axis=1)
    weights = np.stack([s_in[p0], s_in[p1], s_out[p0], s_out[p1]], axis=1)
    band = AirGap(nodes=nodes, weights=weights, inner_radius_m=0.045, outer_radius_m=0.046,
                  arc_length_deg=180.0 if sector else 360.0, inner_shift=float(inner_shift),
                  outer_shift=float(outer_shift), antiperiodic=sector)
    return Model(
        xy=xy, tri=tri, tri_mat=mat,
        nu0=([nu_air, nu_air, nu_air / 1.05, nu_air] + [nu_air] * 6)[:M],
        alpha=np.zeros(M),
        j_per_a=([0.0, 0.0, 0.0, 0.0] + jpa + [-v for v in jpa])[:M],
        hc=([0.0, 0.0, hc] + [0.0] * 7)[:M],
        mag_deg=([0.0, 0.0, 90.0 + rotor_deg] + [0.0] * 7)[:M],
        curve_index=([-1, 0, -1, 0] + [-1] * 6)[:M],
        circuit_index=[-1, -1, -1, -1, 0, 1, 2, 0, 1, 2][:M],
        group=[50, 20, 20, 30, 40, 41, 42, 40, 41, 42][:M],
        curves=[(b_t, hh)],
        dir_nodes=outer, dir_values=np.zeros(outer.size),
        con_a=con_a, con_b=con_b, con_sign=np.full(con_a.size, -1, np.int8),
        circuit_count=3, depth_m=0.05, problem_type=PLANAR,
        name=f"sliding_band_{'sector' if sector else 'full'}_{nr}x{nt}_{rotor_deg:g}deg", ages=[band],
    )
