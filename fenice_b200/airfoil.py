"""Unit sections of airfoil bodies for the immersed boundary: the NACA 4-digit family and coordinate files, as the
reference builds them (naca4, naca_digits and load_airfoil, cpp/src/Geometry.cpp:40-141). A section is a list of (x, y)
vertices with the leading edge at the origin and chord 1 along x; the library places it (place_airfoil). The arithmetic
is the reference's with the C library's functions (Python's math module calls them), so the vertices carry its bits.
"""
import math
import re

_PI = 3.14159265358979323846


def naca_digits(shape):
    """The four digits of a 'NACA dddd' shape name ('' for another name)."""
    s = "".join(ch.lower() for ch in str(shape) if not ch.isspace())
    if len(s) != 8 or not s.startswith("naca") or not s[4:].isdigit():
        return ""
    return s[4:]


def naca4(digits, n=200):
    """The NACA 4-digit section with n + 1 cosine-spaced stations per surface and a closed trailing edge: the upper
    surface from the trailing edge to the leading edge, then the lower surface back (the trailing edge shared)."""
    if len(digits) != 4 or not digits.isdigit():
        raise ValueError(f"NACA 4-digit code must be 4 digits, got '{digits}'")
    m, p = int(digits[0]) / 100.0, int(digits[1]) / 10.0
    t = int(digits[2:]) / 100.0
    if not t > 0.0:
        raise ValueError(f"NACA {digits}: zero thickness")
    if m > 0.0 and not p > 0.0:
        raise ValueError(f"NACA {digits}: camber needs a camber position")
    up, lo = [], []
    for i in range(n + 1):
        x = 0.5 * (1.0 - math.cos(_PI * i / n))
        yt = 5.0 * t * (0.2969 * math.sqrt(x) - 0.1260 * x - 0.3516 * x * x + 0.2843 * x * x * x - 0.1036 * x * x * x * x)
        yc = dyc = 0.0
        if m > 0.0:
            if x < p:
                yc = m / (p * p) * (2.0 * p * x - x * x)
                dyc = 2.0 * m / (p * p) * (p - x)
            else:
                yc = m / ((1 - p) * (1 - p)) * (1.0 - 2.0 * p + 2.0 * p * x - x * x)
                dyc = 2.0 * m / ((1 - p) * (1 - p)) * (p - x)
        th = math.atan(dyc)
        up.append((x - yt * math.sin(th), yc + yt * math.cos(th)))
        lo.append((x + yt * math.sin(th), yc - yt * math.cos(th)))
    return [up[i] for i in range(n, -1, -1)] + [lo[i] for i in range(1, n)]


_NUM = re.compile(r"\s*([+-]?(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?)")


def _pair(line):
    """'x y' at the start of a line (more text after them ignored), as two strtod calls read them; None otherwise."""
    a = _NUM.match(line)
    if not a:
        return None
    b = _NUM.match(line, a.end())
    if not b:
        return None
    return float(a.group(1)), float(b.group(1))


def load_airfoil(path):
    """A Selig or Lednicer coordinate file: an optional name line, (Lednicer) the two point counts, then 'x y' rows;
    normalised to the leading edge at the origin and chord 1."""
    with open(path) as f:
        lines = [(no, text) for no, text in enumerate(f.read().split("\n"), 1) if text.strip(" \t\r")]
    k = 0
    if lines and _pair(lines[0][1]) is None:
        k = 1   # name line
    lednicer, n_up, n_lo = False, 0, 0
    if k < len(lines):
        ab = _pair(lines[k][1])
        if ab is not None and ab[0] > 1.0 and ab[1] > 1.0:
            lednicer, n_up, n_lo = True, int(ab[0]), int(ab[1])
            k += 1
    data = []
    for no, text in lines[k:]:
        ab = _pair(text)
        if ab is None:
            raise ValueError(f"{path}:{no}: expected 'x y', got '{text}'")
        data.append(ab)
    if lednicer:
        if len(data) != n_up + n_lo:
            raise ValueError(f"{path}: Lednicer header announces {n_up} + {n_lo} points, the file has {len(data)}")
        pts = [data[i] for i in range(n_up - 1, -1, -1)] + [data[i] for i in range(n_up, n_up + n_lo) if i > n_up or data[i] != data[0]]
    else:
        pts = list(data)
    if len(pts) > 1 and pts[0] == pts[-1]:
        pts.pop()
    if len(pts) < 3:
        raise ValueError(f"{path}: an airfoil needs at least 3 points")
    x0, y0 = min(pts, key=lambda q: q[0])   # the first of the smallest x
    xmax = x0
    for q in pts:
        xmax = max(xmax, q[0])
    c = xmax - x0
    if not c > 0.0:
        raise ValueError(f"{path}: the coordinates have zero chord")
    return [((x - x0) / c, (y - y0) / c) for x, y in pts]
