"""Pure-Python restatement of llg-sim's OVF 2.0 writers (ovf.rs:54-251).

TEST INFRASTRUCTURE ONLY: the checker of the library's OVF writers.  The
number format is Rust's `{:.<p>e}` (correctly rounded mantissa, ties to even,
exponent without sign padding), produced here with exact decimal arithmetic.
"""
import math
import struct
from decimal import ROUND_HALF_EVEN, Decimal

import numpy as np


def rust_exp(v, prec):
    v = float(v)
    if math.isnan(v):
        return "NaN"
    if math.isinf(v):
        return "inf" if v > 0 else "-inf"
    sign = "-" if math.copysign(1.0, v) < 0 else ""
    d = Decimal(abs(v))                       # exact value of the double
    if d == 0:
        return sign + ("0." + "0" * prec if prec else "0") + "e0"
    exp = d.adjusted()
    quantum = Decimal(1).scaleb(-prec)
    q = d.scaleb(-exp).quantize(quantum, rounding=ROUND_HALF_EVEN)
    if q >= 10:
        exp += 1
        q = d.scaleb(-exp).quantize(quantum, rounding=ROUND_HALF_EVEN)
    return f"{sign}{q:.{prec}f}e{exp}"


def _lines(*ls):
    return "".join(x + "\n" for x in ls).encode()


def ovf2_text_bytes(nx, ny, dx, dy, dz, m, title, desc, labels, units):
    """write_ovf2_rectangular_text (ovf.rs:54-151)."""
    e16 = lambda x: rust_exp(x, 16)
    out = _lines("# OOMMF OVF 2.0", "# Segment count: 1", "# Begin: Segment", "# Begin: Header",
                 f"# Title: {title}", "# meshtype: rectangular", "# meshunit: m",
                 f"# xmin: {e16(0.0)}", f"# ymin: {e16(0.0)}", f"# zmin: {e16(0.0)}",
                 f"# xmax: {e16(nx * dx)}", f"# ymax: {e16(ny * dy)}", f"# zmax: {e16(1 * dz)}",
                 "# valuedim: 3", "# valuelabels: " + " ".join(labels), "# valueunits: " + " ".join(units),
                 *[f"# Desc: {d}" for d in desc],
                 f"# xbase: {e16(0.5 * dx)}", f"# ybase: {e16(0.5 * dy)}", f"# zbase: {e16(0.5 * dz)}",
                 f"# xnodes: {nx}", f"# ynodes: {ny}", "# znodes: 1",
                 f"# xstepsize: {e16(dx)}", f"# ystepsize: {e16(dy)}", f"# zstepsize: {e16(dz)}",
                 "# End: Header", "# Begin: Data Text")
    body = "".join(f"{rust_exp(v[0], 10)} {rust_exp(v[1], 10)} {rust_exp(v[2], 10)}\n" for v in m)
    return out + body.encode() + _lines("# End: Data Text", "# End: Segment")


def ovf2_binary4_bytes(nx, ny, dx, dy, dz, m, title, desc, labels, units):
    """write_ovf2_rectangular_binary4 (ovf.rs:153-251)."""
    e17 = lambda x: rust_exp(x, 17)
    out = _lines("# OOMMF OVF 2.0", "# Segment count: 1", "# Begin: Segment", "# Begin: Header",
                 f"# Title: {title}", *[f"# Desc: {d}" for d in desc], "# meshunit: m", "# meshtype: rectangular",
                 f"# xbase: {e17(0.5 * dx)}", f"# ybase: {e17(0.5 * dy)}", f"# zbase: {e17(0.5 * dz)}",
                 f"# xstepsize: {e17(dx)}", f"# ystepsize: {e17(dy)}", f"# zstepsize: {e17(dz)}",
                 f"# xnodes: {nx}", f"# ynodes: {ny}", "# znodes: 1",
                 "# xmin: 0", f"# xmax: {e17(nx * dx)}", "# ymin: 0", f"# ymax: {e17(ny * dy)}",
                 "# zmin: 0", f"# zmax: {e17(dz)}",
                 "# valuedim: 3", "# valuelabels: " + " ".join(labels), "# valueunits: " + " ".join(units),
                 "# End: Header", "# Begin: Data Binary 4")
    # `v as f32`: round to nearest even, out of range -> +-inf (numpy's conversion does the same)
    with np.errstate(over="ignore"):
        data = np.asarray(m, dtype=np.float64).reshape(-1).astype("<f4").tobytes()
    payload = struct.pack("<f", 1234567.0) + data
    return out + payload + _lines("", "# End: Data Binary 4", "# End: Segment", "# End: File")
