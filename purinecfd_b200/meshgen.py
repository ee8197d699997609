"""O-mesh generators and the O-mesh text format.

The solver reads the reference's text format (jst-rs/src/mesh.rs:1-12)::

    n_rings n_theta
    x y            <- ring by ring (ring 0 = wall), counter-clockwise within a ring

Generators (all off the hot path, used to make inputs):

* ``ellipse_o_mesh`` — the reference's ellipse-cylinder family (wall ellipse with
  semi-axes (a, b), far-field circle of radius r_far, radial parameter spaced
  uniformly or geometrically).  With the defaults and (10, 12) it produces the
  reference's ``fangdata.txt``; with (17, 40, stretch=1.12) its
  ``meshes/cyl_17x40.txt`` (same printed digits).
* ``cylinder_o_mesh`` — a circular cylinder with a geometric radial distribution
  set by the first wall spacing and the far-field radius.
* ``naca4_o_mesh`` — an algebraic O-mesh around a NACA 4-digit section (closed
  trailing edge), cosine-clustered along the surface, geometric radial
  stretching from a given wall spacing, wall-normal extrusion near the wall
  blended into straight lines to a far-field circle.
"""

from __future__ import annotations

import math
from pathlib import Path

import numpy as np


def _geometric_params(n_rings: int, stretch: float) -> list[float]:
    """Normalised radial parameter s in [0, 1] with ring widths stretch**k."""
    if abs(stretch - 1.0) < 1e-12:
        return [i / (n_rings - 1) for i in range(n_rings)]
    widths = [stretch ** k for k in range(n_rings - 1)]
    total = 0.0
    for w in widths:
        total += w
    out, acc = [0.0], 0.0
    for w in widths:
        acc += w
        out.append(acc / total)
    return out


def ellipse_o_mesh(n_rings: int, n_theta: int, a_wall: float = 1.0, b_wall: float = 0.5,
                   r_far: float = 5.0, stretch: float = 1.0) -> np.ndarray:
    """Ellipse wall -> circular far field.  Returns nodes [n_rings*n_theta, 2] (open rings)."""
    if n_rings < 4 or n_theta < 8:
        raise ValueError("an O-mesh needs at least 4 rings and 8 points per ring")
    if stretch <= 0:
        raise ValueError("stretch must be > 0")
    pts = np.empty((n_rings * n_theta, 2))
    k = 0
    for s in _geometric_params(n_rings, stretch):
        a = a_wall + s * (r_far - a_wall)
        b = b_wall + s * (r_far - b_wall)
        for j in range(n_theta):
            th = 2.0 * math.pi * j / n_theta
            pts[k, 0] = a * math.cos(th)
            pts[k, 1] = b * math.sin(th)
            k += 1
    return pts


def geometric_ratio(first: float, total: float, n_intervals: int) -> float:
    """Ratio q with first*(q**n - 1)/(q - 1) == total (bisection in log space, q >= 1)."""
    if first * n_intervals >= total:
        return 1.0

    def log_sum(q):  # log(first * (q**n - 1) / (q - 1)) without overflow
        a = n_intervals * math.log(q)
        return math.log(first) + a + math.log(-math.expm1(-a)) - math.log(q - 1.0)

    target = math.log(total)
    lo, hi = 1.0 + 1e-12, 2.0
    while log_sum(hi) < target:
        hi *= 2.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if log_sum(mid) < target:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def _radial_params(n_rings: int, first_frac: float) -> np.ndarray:
    """s_k = first_frac*(q**k - 1)/(q - 1), s_0 = 0, s_{n-1} = 1."""
    n = n_rings - 1
    q = geometric_ratio(first_frac, 1.0, n)
    if q == 1.0:
        return np.linspace(0.0, 1.0, n_rings)
    k = np.arange(n_rings, dtype=np.float64)
    s = first_frac * (q ** k - 1.0) / (q - 1.0)
    s[-1] = 1.0
    return s


def cylinder_o_mesh(n_rings: int, n_theta: int, radius: float = 0.5, r_far: float = 20.0,
                    first_spacing: float = 1e-3) -> np.ndarray:
    """Circular cylinder O-mesh with geometric radial spacing.  Open rings, CCW."""
    if n_rings < 4 or n_theta < 8:
        raise ValueError("an O-mesh needs at least 4 rings and 8 points per ring")
    s = _radial_params(n_rings, first_spacing / (r_far - radius))
    r = radius + s * (r_far - radius)
    th = 2.0 * np.pi * np.arange(n_theta) / n_theta
    x = r[:, None] * np.cos(th)[None, :]
    y = r[:, None] * np.sin(th)[None, :]
    return np.stack([x.ravel(), y.ravel()], axis=1)


def naca4_surface(phi: np.ndarray, m: float, p: float, t: float, chord: float = 1.0):
    """Points on a NACA 4-digit section (closed trailing edge) at surface angle phi.

    phi = 0 is the trailing edge, phi in (0, pi) the upper surface (TE -> LE),
    phi = pi the leading edge and phi in (pi, 2pi) the lower surface, so that
    increasing phi runs counter-clockwise.  x = 0.5*(1 + cos(phi)) clusters
    points at both edges."""
    x = 0.5 * (1.0 + np.cos(phi))
    yt = 5.0 * t * (0.2969 * np.sqrt(np.maximum(x, 0.0)) - 0.1260 * x - 0.3516 * x ** 2
                    + 0.2843 * x ** 3 - 0.1036 * x ** 4)
    if m > 0.0 and p > 0.0:
        fore = x < p
        yc = np.where(fore, m / p ** 2 * (2 * p * x - x ** 2), m / (1 - p) ** 2 * ((1 - 2 * p) + 2 * p * x - x ** 2))
        dyc = np.where(fore, 2 * m / p ** 2 * (p - x), 2 * m / (1 - p) ** 2 * (p - x))
    else:
        yc = np.zeros_like(x)
        dyc = np.zeros_like(x)
    th = np.arctan(dyc)
    upper = np.sin(phi) >= 0.0
    sgn = np.where(upper, 1.0, -1.0)
    xs = x - sgn * yt * np.sin(th)
    ys = yc + sgn * yt * np.cos(th)
    return chord * xs, chord * ys


def _wall_normals(wx: np.ndarray, wy: np.ndarray, smooth: int) -> tuple[np.ndarray, np.ndarray]:
    """Unit outward normals of a closed counter-clockwise wall polyline,
    from central differences, then `smooth` passes of neighbour averaging
    (periodic), which turns the normals gradually round a sharp trailing edge."""
    tx = np.roll(wx, -1) - np.roll(wx, 1)
    ty = np.roll(wy, -1) - np.roll(wy, 1)
    nx, ny = ty, -tx
    ln = np.hypot(nx, ny)
    nx, ny = nx / ln, ny / ln
    for _ in range(smooth):
        nx = 0.25 * np.roll(nx, 1) + 0.5 * nx + 0.25 * np.roll(nx, -1)
        ny = 0.25 * np.roll(ny, 1) + 0.5 * ny + 0.25 * np.roll(ny, -1)
        ln = np.hypot(nx, ny)
        nx, ny = nx / ln, ny / ln
    return nx, ny


def naca4_o_mesh(n_rings: int, n_theta: int, m: float = 0.0, p: float = 0.4, t: float = 0.12,
                 chord: float = 1.0, r_far: float = 30.0, first_spacing: float = 1e-6,
                 orthogonal: bool = True, smooth: int = 8) -> np.ndarray:
    """O-mesh around a NACA 4-digit section.  Open rings, CCW, ring 0 = wall.

    m, p, t are the camber, camber position and thickness as fractions of the
    chord (NACA 2412 -> m=0.02, p=0.4, t=0.12).  The far field is a circle of
    radius r_far*chord around mid-chord.  Rings are placed at the geometric
    radial parameter s_i (first step first_spacing*chord over the nominal
    distance).  With `orthogonal`, node (i, j) blends a wall-normal extrusion
    w_j + d_i n_j (smoothed normals, d_i the radial distance) with the straight
    line from wall point j to far-field point j, weighted by s_i, so the wall
    cells are nearly orthogonal and the trailing-edge cells are not slivers;
    otherwise only the straight lines are used."""
    if n_rings < 4 or n_theta < 8:
        raise ValueError("an O-mesh needs at least 4 rings and 8 points per ring")
    phi = 2.0 * np.pi * np.arange(n_theta) / n_theta
    wx, wy = naca4_surface(phi, m, p, t, chord)
    cx = 0.5 * chord
    fx = cx + r_far * chord * np.cos(phi)
    fy = r_far * chord * np.sin(phi)
    length = (r_far - 0.5) * chord
    s = _radial_params(n_rings, first_spacing * chord / length)
    bx = wx[None, :] + s[:, None] * (fx - wx)[None, :]
    by = wy[None, :] + s[:, None] * (fy - wy)[None, :]
    if orthogonal:
        nx, ny = _wall_normals(wx, wy, smooth)
        d = s * length
        ax = wx[None, :] + d[:, None] * nx[None, :]
        ay = wy[None, :] + d[:, None] * ny[None, :]
        wgt = np.sqrt(s)[:, None]
        x = (1.0 - wgt) * ax + wgt * bx
        y = (1.0 - wgt) * ay + wgt * by
    else:
        x, y = bx, by
    return np.stack([x.ravel(), y.ravel()], axis=1)


def close_rings(pts: np.ndarray, n_rings: int, n_theta: int) -> np.ndarray:
    """Append each ring's first point at its end (the closed-ring file form)."""
    r = pts.reshape(n_rings, n_theta, 2)
    return np.concatenate([r, r[:, :1, :]], axis=1).reshape(-1, 2)


def format_mesh(pts: np.ndarray, n_rings: int, n_theta: int, digits: int = 10) -> str:
    """The reference's text format: header then one `x y` per line."""
    fmt = f"{{:.{digits}f}} {{:.{digits}f}}\n"
    return f"{n_rings} {n_theta}\n" + "".join(fmt.format(x, y) for x, y in pts)


def write_mesh(path: str | Path, pts: np.ndarray, n_rings: int, n_theta: int, digits: int = 10) -> None:
    Path(path).parent.mkdir(parents=True, exist_ok=True)
    Path(path).write_text(format_mesh(pts, n_rings, n_theta, digits), encoding="utf-8")
