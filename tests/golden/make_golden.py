"""Generates the golden fixtures in this directory (run: python tests/golden/make_golden.py).

The values are computed here in pure Python, independently of the C++ oracle
and of the CUDA library, by restating:
  - XorShift64 and its [0,1) mapping (initial_states.rs:230-254);
  - the MuMax-like face-charge integration of the demag kernel,
    kernel_2d_components_mumax_like / mumax_like_h_from_unit_m
    (demag_fft_uniform.rs:1076-1253), same loop order and rounding order.
The tests check the oracle (and through it the GPU path) against them.
"""
import json
import math
import os

HERE = os.path.dirname(os.path.abspath(__file__))
PI = math.pi
MU0 = 4.0 * PI * 1e-7
M64 = (1 << 64) - 1


def xorshift_f64(seed, count):
    s = 0x9E3779B97F4A7C15 if seed == 0 else seed
    out = []
    for _ in range(count):
        s ^= (s << 13) & M64
        s ^= s >> 7
        s ^= (s << 17) & M64
        out.append(float(s >> 11) * (1.0 / float(1 << 53)))
    return out


def _mumax_n(x):
    return int(math.floor(max(x, 1.0) + 0.5))


def _delta_cell(d):
    a = float(abs(d))
    return a - 1.0 if a > 0.0 else a


def h_from_unit_m(u, rc, cell, disp, accuracy):
    v, w = (u + 1) % 3, (u + 2) % 3
    lmin = min(cell[0], cell[1], cell[2])
    dxm, dym, dzm = (_delta_cell(disp[k]) * cell[k] for k in range(3))
    d = math.sqrt(dxm * dxm + dym * dym + dzm * dzm)
    if d == 0.0:
        d = lmin
    max_size = d / accuracy
    nx, ny, nz = (_mumax_n(cell[k] / max_size) for k in range(3))
    nv = 2 * _mumax_n(cell[v] / max_size)
    nw = 2 * _mumax_n(cell[w] / max_size)
    scale = 1.0 / float(nv * nw * nx * ny * nz)
    charge = cell[v] * cell[w] * scale
    pu1 = 0.5 * cell[u]
    pu2 = -pu1
    pole = [0.0, 0.0, 0.0]
    h = [0.0, 0.0, 0.0]
    for i in range(nv):
        pole[v] = -0.5 * cell[v] + cell[v] / (2.0 * nv) + i * (cell[v] / nv)
        for j in range(nw):
            pole[w] = -0.5 * cell[w] + cell[w] / (2.0 * nw) + j * (cell[w] / nw)
            for ax in range(nx):
                rx = rc[0] - 0.5 * cell[0] + cell[0] / (2.0 * nx) + ax * (cell[0] / nx)
                for ay in range(ny):
                    ry = rc[1] - 0.5 * cell[1] + cell[1] / (2.0 * ny) + ay * (cell[1] / ny)
                    for az in range(nz):
                        rz = rc[2] - 0.5 * cell[2] + cell[2] / (2.0 * nz) + az * (cell[2] / nz)
                        pole[u] = pu1
                        r1x, r1y, r1z = rx - pole[0], ry - pole[1], rz - pole[2]
                        r1 = math.sqrt(r1x * r1x + r1y * r1y + r1z * r1z)
                        q1 = charge / (4.0 * PI * r1 * r1 * r1)
                        pole[u] = pu2
                        r2x, r2y, r2z = rx - pole[0], ry - pole[1], rz - pole[2]
                        r2 = math.sqrt(r2x * r2x + r2y * r2y + r2z * r2z)
                        q2 = -charge / (4.0 * PI * r2 * r2 * r2)
                        h[0] += r1x * q1 + r2x * q2
                        h[1] += r1y * q1 + r2y * q2
                        h[2] += r1z * q1 + r2z * q2
    return h


def kernel_components(dx, dy, dz, sx, sy, accuracy=10.0):
    rc = [sx * dx, sy * dy, 0.0]
    cell = [dx, dy, dz]
    disp = [sx, sy, 0]
    hx = h_from_unit_m(0, rc, cell, disp, accuracy)
    hy = h_from_unit_m(1, rc, cell, disp, accuracy)
    hz = h_from_unit_m(2, rc, cell, disp, accuracy)
    return [MU0 * hx[0], MU0 * hy[0], MU0 * hy[1], MU0 * hz[2]]


CELLS = [(4e-9, 4e-9, 3e-9), (2e-9, 2e-9, 2e-9), (5e-9, 4e-9, 1e-9)]
DISPS = [(0, 0), (1, 0), (0, 1), (1, 1), (2, 3), (5, 0), (7, 0), (8, 3), (20, 1), (40, 40)]


def main():
    xs = {str(seed): xorshift_f64(seed, 32) for seed in (0, 1, 7, 12345, 0xDEADBEEF)}
    with open(os.path.join(HERE, "xorshift_f64.json"), "w") as f:
        json.dump(xs, f, indent=1)
    kc = []
    for cell in CELLS:
        for (sx, sy) in DISPS:
            kc.append({"cell": list(cell), "sx": sx, "sy": sy, "k": kernel_components(*cell, sx, sy)})
    with open(os.path.join(HERE, "kernel_components.json"), "w") as f:
        json.dump(kc, f, indent=1)


if __name__ == "__main__":
    main()
