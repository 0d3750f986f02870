"""Seeded synthetic UVLM workloads: wing and body meshes plus their kinematics.

The reference ships no benchmark geometry; these generators produce seeded
stand-ins with the shapes, sizes and motions of the five workloads the solver is
measured on:

* ``flat_wing``     -- 16 x 4 flat rectangular wing, AR 8, static, 10 free-wake steps.
* ``swept_pitching``-- 64 x 16 swept (25 deg), tapered (0.5) wing, cosine spanwise
  spacing, pitching about the root quarter chord, 200 steps.
* ``icosphere``     -- closed unit sphere of 5120 triangles with N(0, 1e-3) node jitter.
* ``batch_wings``   -- 256 independent wings of 128..2048 rings (log-uniform).
* ``flapping``      -- 128 x 32 heaving, twisting, bending wing, wake cut at 400 rows.

A workload is a :class:`Case`: body node positions in the body frame, element
connectivity (vortex-ring vertex loops), the trailing-edge node pairs that shed
wake, and a :class:`Kinematics` giving global positions and velocities at time t.
Element loops are ordered so that the reference's ring normal
(src/core/mesh.c:48-68) points to +z on a flat wing.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import numpy.typing as npt


# --------------------------------------------------------------------------- kinematics
class Kinematics:
    """Maps body-frame node positions to global positions and velocities at time t."""

    def positions(self, pos0: npt.NDArray[np.float64], t: float) -> npt.NDArray[np.float64]:
        raise NotImplementedError

    def velocities(self, pos0: npt.NDArray[np.float64], t: float) -> npt.NDArray[np.float64]:
        raise NotImplementedError


class Static(Kinematics):
    """No motion: positions are the body-frame positions, velocities are zero."""

    def positions(self, pos0, t):
        return np.array(pos0, np.float64)

    def velocities(self, pos0, t):
        return np.zeros_like(pos0, dtype=np.float64)


def _rot_y(phi: float | npt.NDArray) -> tuple:
    return np.cos(phi), np.sin(phi)


@dataclass
class Pitching(Kinematics):
    """Rigid pitch about the spanwise axis through ``(x_pivot, 0, 0)``.

    alpha(t) = alpha0 + amp * sin(2 pi k t); a point r maps to
    x = xp + cos(a)(x0 - xp) + sin(a) z0,  z = -sin(a)(x0 - xp) + cos(a) z0,
    so a positive angle lowers the trailing edge (nose up).
    """

    alpha0: float
    amp: float
    k: float
    x_pivot: float

    def alpha(self, t):
        return self.alpha0 + self.amp * np.sin(2 * np.pi * self.k * t)

    def alpha_dot(self, t):
        return self.amp * 2 * np.pi * self.k * np.cos(2 * np.pi * self.k * t)

    def positions(self, pos0, t):
        c, s = _rot_y(self.alpha(t))
        dx = pos0[:, 0] - self.x_pivot
        z0 = pos0[:, 2]
        out = np.empty_like(pos0, dtype=np.float64)
        out[:, 0] = self.x_pivot + c * dx + s * z0
        out[:, 1] = pos0[:, 1]
        out[:, 2] = -s * dx + c * z0
        return out

    def velocities(self, pos0, t):
        c, s = _rot_y(self.alpha(t))
        ad = self.alpha_dot(t)
        dx = pos0[:, 0] - self.x_pivot
        z0 = pos0[:, 2]
        out = np.zeros_like(pos0, dtype=np.float64)
        out[:, 0] = ad * (-s * dx + c * z0)
        out[:, 2] = ad * (-c * dx - s * z0)
        return out


@dataclass
class Flapping(Kinematics):
    """Heave + spanwise-linear twist + quadratic bending of a wing lying in z = 0.

    With w = omega t, s = y / semi_span in [-1, 1]:
      theta(y, t) = twist * |s| * cos(w)                (twist about x = x_pivot)
      z_shift(y, t) = heave * sin(w) + bend * s^2 * sin(w)
      x = xp + cos(theta)(x0 - xp);  z = -sin(theta)(x0 - xp) + z_shift
    """

    omega: float
    heave: float
    twist: float
    bend: float
    semi_span: float
    x_pivot: float

    def _parts(self, pos0, t):
        w = self.omega * t
        s = pos0[:, 1] / self.semi_span
        theta = self.twist * np.abs(s) * np.cos(w)
        theta_dot = -self.twist * np.abs(s) * np.sin(w) * self.omega
        zs = (self.heave + self.bend * s * s) * np.sin(w)
        zs_dot = (self.heave + self.bend * s * s) * np.cos(w) * self.omega
        return theta, theta_dot, zs, zs_dot

    def positions(self, pos0, t):
        theta, _, zs, _ = self._parts(pos0, t)
        dx = pos0[:, 0] - self.x_pivot
        out = np.empty_like(pos0, dtype=np.float64)
        out[:, 0] = self.x_pivot + np.cos(theta) * dx
        out[:, 1] = pos0[:, 1]
        out[:, 2] = -np.sin(theta) * dx + zs + pos0[:, 2]
        return out

    def velocities(self, pos0, t):
        theta, theta_dot, _, zs_dot = self._parts(pos0, t)
        dx = pos0[:, 0] - self.x_pivot
        out = np.zeros_like(pos0, dtype=np.float64)
        out[:, 0] = -np.sin(theta) * theta_dot * dx
        out[:, 2] = -np.cos(theta) * theta_dot * dx + zs_dot
        return out


# --------------------------------------------------------------------------- cases
@dataclass
class Case:
    """One UVLM workload: topology, body-frame positions, motion, flow and run length."""

    name: str
    positions: npt.NDArray[np.float64]          # (n_points, 3) body frame
    elements: list[npt.NDArray[np.uint32]]      # vertex loops, one per ring
    kinematics: Kinematics
    freestream: npt.NDArray[np.float64]          # (3,) uniform U_inf
    dt: float
    nt: int
    line_rows: int                               # wake rows kept (0 = no wake)
    te_node_pairs: npt.NDArray[np.uint32]        # (S, 2) node pairs of shedding lines
    closed: bool = False
    tol: float = 1e-6
    s_ref: float = 1.0                           # reference area for CL
    t0: float = 0.0                              # wake model start time (first dt)
    meta: dict = field(default_factory=dict)
    # (ring0, n_span, n_chord) blocks of rings ring0 + i * n_chord + j over which the control
    # points are smooth in (i, j) (MixedSolverEngine cp_patches); empty: not a structured grid
    smooth_patches: tuple = ()
    # (col0, n) runs of wake node columns (trailing-edge nodes, in the engine's de-duplicated
    # column order) along which the wake is smooth (MixedSolverEngine wake_col_runs)
    wake_col_runs: tuple = ()

    @property
    def n_points(self) -> int:
        return int(self.positions.shape[0])

    @property
    def n_surfaces(self) -> int:
        return len(self.elements)

    def positions_at(self, t: float) -> npt.NDArray[np.float64]:
        return self.kinematics.positions(self.positions, t)

    def velocities_at(self, t: float) -> npt.NDArray[np.float64]:
        return self.kinematics.velocities(self.positions, t)

    def lift_direction(self) -> npt.NDArray[np.float64]:
        """Unit vector normal to U_inf in the x-z plane (CL direction)."""
        u = self.freestream
        l = np.array([-u[2], 0.0, u[0]], np.float64)
        return l / np.linalg.norm(l)


def _grid_wing(xs: npt.NDArray, ys: npt.NDArray) -> tuple:
    """Structured quad grid; xs is (ns+1, nc+1) chordwise coords, ys (ns+1,) spanwise.

    Node (i, j) = i * (nc + 1) + j; ring (i, j) = i * nc + j with the loop
    (i,j) -> (i+1,j) -> (i+1,j+1) -> (i,j+1) whose reference normal is +z.
    Returns positions, elements and the trailing-edge node pairs (j = nc).
    """
    ns1, nc1 = xs.shape
    ns, nc = ns1 - 1, nc1 - 1
    pos = np.zeros((ns1 * nc1, 3), np.float64)
    pos[:, 0] = xs.reshape(-1)
    pos[:, 1] = np.repeat(ys, nc1)
    i, j = np.meshgrid(np.arange(ns), np.arange(nc), indexing="ij")
    n00 = (i * nc1 + j).reshape(-1)
    loops = np.stack([n00, n00 + nc1, n00 + nc1 + 1, n00 + 1], axis=1).astype(np.uint32)
    te = np.stack([np.arange(ns) * nc1 + nc, (np.arange(ns) + 1) * nc1 + nc], axis=1)
    return pos, [loops[k] for k in range(loops.shape[0])], te.astype(np.uint32)


def _root_split(ns: int, nc: int) -> tuple:
    """The two half wings of a _grid_wing whose shape or motion depends on |y| (a kink at the
    root, y = 0, between strips ns/2 - 1 and ns/2); one patch for an odd strip count."""
    if ns % 2:
        return ((0, ns, nc),)
    h = ns // 2
    return ((0, h, nc), (h * nc, h, nc))


def _root_split_cols(ns: int) -> tuple:
    """The trailing-edge node columns of _root_split's halves (sharing the root node ns/2)."""
    if ns % 2:
        return ((0, ns + 1),)
    h = ns // 2
    return ((0, h + 1), (h, h + 1))


def flat_wing(ns: int = 16, nc: int = 4, span: float = 8.0, chord: float = 1.0,
              alpha_deg: float = 5.0, dt: float = 0.25, nt: int = 10,
              line_rows: int = 10) -> Case:
    """Flat rectangular wing in the xy-plane, uniform spacing, static, U_inf at alpha."""
    x = np.linspace(0.0, chord, nc + 1)
    y = np.linspace(-span / 2, span / 2, ns + 1)
    xs = np.broadcast_to(x, (ns + 1, nc + 1)).copy()
    pos, elements, te = _grid_wing(xs, y)
    a = np.radians(alpha_deg)
    return Case(
        name=f"flat_wing_{ns}x{nc}",
        positions=pos, elements=elements, kinematics=Static(),
        freestream=np.array([np.cos(a), 0.0, np.sin(a)]), dt=dt, nt=nt,
        line_rows=line_rows, te_node_pairs=te, s_ref=span * chord, t0=-dt,
    )


def swept_pitching(ns: int = 64, nc: int = 16, seed: int = 1, span: float = 8.0,
                   root_chord: float = 1.0, sweep_deg: float = 25.0, taper: float = 0.5,
                   nt: int = 200, line_rows: int = 200, dt: float | None = None) -> Case:
    """Swept, tapered wing with cosine spanwise spacing pitching about the root c/4.

    alpha(t) = 5 deg + 3 deg sin(2 pi k t), k ~ U[0.05, 0.3] from ``seed``;
    U_inf = (1, 0, 0); dt defaults to root_chord / nc.
    """
    rng = np.random.default_rng(seed)
    k = float(rng.uniform(0.05, 0.3))
    half = span / 2
    y = -half * np.cos(np.pi * np.arange(ns + 1) / ns)
    y[np.abs(y) < 1e-15] = 0.0
    eta = np.abs(y) / half
    chord = root_chord * (1.0 - (1.0 - taper) * eta)
    x_le = np.abs(y) * np.tan(np.radians(sweep_deg))
    xs = x_le[:, None] + chord[:, None] * np.linspace(0.0, 1.0, nc + 1)[None, :]
    pos, elements, te = _grid_wing(xs, y)
    dt = root_chord / nc if dt is None else dt
    kin = Pitching(alpha0=np.radians(5.0), amp=np.radians(3.0), k=k, x_pivot=0.25 * root_chord)
    s_ref = span * root_chord * (1 + taper) / 2
    return Case(
        name=f"swept_pitching_{ns}x{nc}",
        positions=pos, elements=elements, kinematics=kin,
        freestream=np.array([1.0, 0.0, 0.0]), dt=dt, nt=nt, line_rows=line_rows,
        te_node_pairs=te, s_ref=s_ref, t0=-dt, meta={"k": k, "seed": seed},
        smooth_patches=_root_split(ns, nc), wake_col_runs=_root_split_cols(ns),
    )


def flapping(ns: int = 128, nc: int = 32, span: float = 8.0, chord: float = 1.0,
             k: float = 0.2, nt: int = 2000, line_rows: int = 400,
             alpha_deg: float = 5.0, dt: float | None = None) -> Case:
    """Rectangular wing heaving 0.2 c, twisting +-10 deg (linear in span), bending ~ y^2.

    omega = 2 k U / c (reduced frequency k); U_inf at alpha; dt defaults to chord / nc.
    """
    x = np.linspace(0.0, chord, nc + 1)
    y = np.linspace(-span / 2, span / 2, ns + 1)
    xs = np.broadcast_to(x, (ns + 1, nc + 1)).copy()
    pos, elements, te = _grid_wing(xs, y)
    a = np.radians(alpha_deg)
    kin = Flapping(omega=2 * k, heave=0.2 * chord, twist=np.radians(10.0),
                   bend=0.1 * chord, semi_span=span / 2, x_pivot=0.25 * chord)
    dt = chord / nc if dt is None else dt
    return Case(
        name=f"flapping_{ns}x{nc}",
        positions=pos, elements=elements, kinematics=kin,
        freestream=np.array([np.cos(a), 0.0, np.sin(a)]), dt=dt, nt=nt,
        line_rows=line_rows, te_node_pairs=te, s_ref=span * chord, t0=-dt,
        meta={"k": k}, smooth_patches=_root_split(ns, nc), wake_col_runs=_root_split_cols(ns),
    )


def _icosphere_base():
    t = (1.0 + 5.0**0.5) / 2.0
    v = np.array([
        [-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0],
        [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
        [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1],
    ], np.float64)
    f = np.array([
        [0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
        [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
        [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
        [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1],
    ], np.int64)
    return v / np.linalg.norm(v, axis=1, keepdims=True), f


def icosphere(subdiv: int = 4, seed: int = 2, jitter: float = 1e-3) -> Case:
    """Unit icosphere, 20 * 4**subdiv triangles, nodes jittered by N(0, jitter^2).

    Steady (one step, no wake); U_inf is a seeded random unit vector.
    """
    rng = np.random.default_rng(seed)
    verts, faces = _icosphere_base()
    verts = list(map(tuple, verts))
    for _ in range(subdiv):
        cache: dict = {}
        new_faces = []

        def mid(a, b):
            key = (a, b) if a < b else (b, a)
            if key not in cache:
                p = (np.array(verts[a]) + np.array(verts[b])) / 2
                verts.append(tuple(p / np.linalg.norm(p)))
                cache[key] = len(verts) - 1
            return cache[key]

        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            new_faces += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = np.array(new_faces, np.int64)
    pos = np.array(verts, np.float64)
    pos += rng.normal(0.0, jitter, pos.shape)
    u = rng.normal(size=3)
    u /= np.linalg.norm(u)
    elements = [np.asarray(f, np.uint32) for f in faces]
    return Case(
        name=f"icosphere_{len(elements)}",
        positions=pos, elements=elements, kinematics=Static(), freestream=u,
        dt=1.0, nt=1, line_rows=0, te_node_pairs=np.zeros((0, 2), np.uint32),
        closed=True, s_ref=np.pi, meta={"seed": seed},
    )


def batch_wings(n_cases: int = 256, seed: int = 3, steps: int = 50,
                p_min: int = 128, p_max: int = 2048) -> list[Case]:
    """Independent swept/tapered wings with log-uniform ring counts in [p_min, p_max].

    Per case: P ~ logU, ns = round(sqrt(4P)), nc = round(P / ns); alpha ~ U[-8, 12] deg,
    sweep ~ U[0, 35] deg, taper ~ U[0.3, 1], AR ~ U[4, 12]; static; ``steps`` free-wake
    steps with a wake of ``steps`` rows.
    """
    rng = np.random.default_rng(seed)
    out = []
    for ic in range(n_cases):
        p = float(np.exp(rng.uniform(np.log(p_min), np.log(p_max))))
        ns = max(2, int(round((4 * p) ** 0.5)))
        nc = max(1, int(round(p / ns)))
        alpha = np.radians(rng.uniform(-8.0, 12.0))
        sweep = rng.uniform(0.0, 35.0)
        taper = rng.uniform(0.3, 1.0)
        ar = rng.uniform(4.0, 12.0)
        root = 1.0
        span = ar * root * (1 + taper) / 2
        half = span / 2
        y = np.linspace(-half, half, ns + 1)
        eta = np.abs(y) / half
        chord = root * (1.0 - (1.0 - taper) * eta)
        x_le = np.abs(y) * np.tan(np.radians(sweep))
        xs = x_le[:, None] + chord[:, None] * np.linspace(0.0, 1.0, nc + 1)[None, :]
        pos, elements, te = _grid_wing(xs, y)
        dt = root / nc
        out.append(Case(
            name=f"batch_{ic}_{ns}x{nc}", positions=pos, elements=elements,
            kinematics=Static(), freestream=np.array([np.cos(alpha), 0.0, np.sin(alpha)]),
            dt=dt, nt=steps, line_rows=steps, te_node_pairs=te,
            s_ref=span * root * (1 + taper) / 2, t0=-dt,
            meta={"alpha": alpha, "sweep": sweep, "taper": taper, "ar": ar},
        ))
    return out


def synthetic_full_wake(te_positions, line_rows: int, freestream, dt: float, seed: int = 0):
    """A seeded, fully developed wake state with every row present.

    te_positions is (S, 2, 3): the two trailing-edge nodes of each shedding line.  Row r
    sits r * dt * U_inf downstream of the trailing edge with a smooth seeded vertical wave;
    circulations are smooth seeded values of the size a lifting wing sheds.  Returns
    positions (S, 2, R+1, 3) and circulations (S, R)."""
    rng = np.random.default_rng(seed)
    te = np.asarray(te_positions, np.float64)
    S, R = te.shape[0], int(line_rows)
    u = np.asarray(freestream, np.float64)
    r = np.arange(R + 1, dtype=np.float64)
    ph = rng.uniform(0, 2 * np.pi)
    pos = te[:, :, None, :] + r[None, None, :, None] * dt * u[None, None, None, :]
    pos[..., 2] += 0.05 * np.sin(0.07 * r + ph)[None, None, :]
    circ = 0.02 * np.sin(0.05 * np.arange(R)[None, :] + np.linspace(0, np.pi, S)[:, None] + ph)
    return pos, circ


def by_name(name: str) -> Case:
    """Workloads by their short names: flat_wing, swept_pitching, icosphere, flapping."""
    table = {
        "flat_wing": flat_wing,
        "swept_pitching": swept_pitching,
        "icosphere": icosphere,
        "flapping": flapping,
    }
    return table[name]()
