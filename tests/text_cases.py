"""Particle CSV texts for the read_csv / write_vtk parity tests: every number
format the reference's parser accepts, and malformed lines."""
import numpy as np

from oracle import PARTICLE


def random_particles(n, seed, special=False):
    """Particles whose doubles span magnitudes from subnormal to huge (and,
    with special, infinities and negative zeros)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(n, PARTICLE)
    p["id"] = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    vals = rng.normal(0, 1, (n, 7)) * 10.0 ** rng.integers(-30, 30, (n, 7))
    tiny = rng.random((n, 7)) < 0.03
    vals[tiny] = rng.random(tiny.sum()) * 1e-310  # subnormals
    big = rng.random((n, 7)) < 0.03
    vals[big] = rng.normal(0, 1, big.sum()) * 1e300
    if special:
        s = rng.random((n, 7))
        vals[s < 0.01] = np.inf
        vals[(s >= 0.01) & (s < 0.02)] = -np.inf
        vals[(s >= 0.02) & (s < 0.03)] = -0.0
    p["mass"] = vals[:, 0]
    p["pos"] = vals[:, 1:4]
    p["vel"] = vals[:, 4:7]
    return p


def _fmt(v, style, rng):
    if style == 0:
        return repr(float(v))  # shortest round trip
    if style == 1:
        return "%.17g" % v
    if style == 2:
        return "%.6e" % v
    if style == 3:
        return "%.25e" % v  # more digits than a double holds
    if style == 4:
        s = "%.17g" % v
        return s.upper()
    if style == 5:  # fixed notation with many digits
        return ("%.40f" % v) if abs(v) < 1e15 else repr(float(v))
    return "%.3g" % v


def csv_text(parts, seed, header=False, crlf=False, blanks=False, blank_lines=False, final_newline=True,
             styles=(0, 1, 2, 3, 4, 5, 6)):
    rng = np.random.default_rng(seed)
    lines = []
    if header:
        lines.append("id,mass,pos_x,pos_y,pos_z,vel_x,vel_y,vel_z")
    for q in parts:
        vals = [q["mass"], *q["pos"], *q["vel"]]
        f = [str(int(q["id"])) if rng.random() < 0.9 else "000" + str(int(q["id"]))]
        f += [_fmt(v, styles[rng.integers(len(styles))], rng) for v in vals]
        if blanks:
            f = [(" " * int(rng.integers(0, 3))) + x + ("\t" if rng.random() < 0.2 else "") for x in f]
        lines.append(",".join(f))
        if blank_lines and rng.random() < 0.05:
            lines.append(" \t" if rng.random() < 0.5 else "")
    sep = "\r\n" if crlf else "\n"
    text = sep.join(lines)
    if final_newline:
        text += sep
    return text.encode()


MALFORMED = [
    b"1,1,2,3,4,5,6\n",                 # seven fields
    b"1,1,2,3,4,5,6,7,8\n",             # nine fields
    b"1,+1,2,3,4,5,6,7\n",              # leading '+'
    b"1,1e,2,3,4,5,6,7\n",              # exponent without digits
    b"1,0x1p3,2,3,4,5,6,7\n",           # hexadecimal
    b"4294967296,1,2,3,4,5,6,7\n",      # id out of range
    b"-1,1,2,3,4,5,6,7\n",              # negative id
    b"1,1e400,2,3,4,5,6,7\n",           # overflow
    b"1,1e-400,2,3,4,5,6,7\n",          # underflow to zero
    b"1,.,2,3,4,5,6,7\n",               # no digits
    b"1,1 2,2,3,4,5,6,7\n",             # blank inside a number
    b"1,1,2,3,4,5,6,7x\n",              # trailing garbage
]
