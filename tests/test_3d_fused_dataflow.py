"""CPU check of the fused 3-D step's data flow (csrc/gb_3d_fused.cuh,
step3_fused_kernel), restated in NumPy float32 CTA by CTA: the z-march over
a chunk, the TMA stages with their zero fill outside the grid, the register
queue of vz planes, the x taps from neighbouring lanes (with the shuffles'
wrap-around in the halo lanes), the ring of 4 new-pressure planes, both
free-surface mirrors, the writes of each CTA's own cells, and the energy
squares summed over a cluster's shots in shot order.

The restatement must equal, bit for bit, a whole-array restatement of the
split kernels (p3_kernel, the mirrors, v3_kernel, in place), which the GPU
tests pin to the reference.  Every cell of the output must be written by
exactly one CTA, and every TMA x coordinate must be a multiple of 4."""
import numpy as np
import pytest

C1, C2 = np.float32(9.0 / 8.0), np.float32(-1.0 / 24.0)
TX, ROW = 120, 128


def d4(a, b, c, d):
    return C1 * (a - b) + C2 * (c - d)   # float32 arrays: every operation rounds to float32


class Geo:
    def __init__(self, nz, ny, nx, pml, S, free_surface):
        self.nz, self.ny, self.nx, self.pml, self.S = nz, ny, nx, pml, S
        self.Nz, self.Ny, self.Nx = nz + 2 * pml, ny + 2 * pml, nx + 2 * pml
        self.pitch = (self.Nx + 31) // 32 * 32
        self.fs = pml if free_surface else 1
        self.free_surface = free_surface


def split_step(g, st, coef, src, amp, energy):
    """p3_kernel, mirror, v3_kernel, mirror on st [S][4][Nz][Ny][pitch], in place."""
    a1, k1, a2, k2, k3, k4 = coef
    one = np.float32(1)
    Nz, Ny, Nx = g.Nz, g.Ny, g.Nx
    z0, z1, y0, y1, x0, x1 = g.fs + 1, Nz - 2, 2, Ny - 2, 2, Nx - 2
    P, VX, VY, VZ = (st[:, f] for f in range(4))
    if z1 > z0 and y1 > y0 and x1 > x0:
        sl = (slice(None), slice(z0, z1), slice(y0, y1), slice(x0, x1))
        dvx = d4(VX[sl], VX[:, z0:z1, y0:y1, x0 - 1:x1 - 1], VX[:, z0:z1, y0:y1, x0 + 1:x1 + 1],
                 VX[:, z0:z1, y0:y1, x0 - 2:x1 - 2])
        dvy = d4(VY[sl], VY[:, z0:z1, y0 - 1:y1 - 1, x0:x1], VY[:, z0:z1, y0 + 1:y1 + 1, x0:x1],
                 VY[:, z0:z1, y0 - 2:y1 - 2, x0:x1])
        dvz = d4(VZ[sl], VZ[:, z0 - 1:z1 - 1, y0:y1, x0:x1], VZ[:, z0 + 1:z1 + 1, y0:y1, x0:x1],
                 VZ[:, z0 - 2:z1 - 2, y0:y1, x0:x1])
        ssum = (dvx + dvy) + dvz
        P[sl] = (one - k1[z0:z1, y0:y1, x0:x1]) * P[sl] - a1[z0:z1, y0:y1, x0:x1] * ssum
    for s in range(g.S):
        P[s, src[s][0], src[s][1], src[s][2]] += amp[s]
    if g.free_surface:
        P[:, g.fs - 1] = -P[:, g.fs + 1]
    pn = P.copy()
    for (F, k, zr, yr, xr, axis) in ((VX, k2, (g.fs, Nz - 1), (1, Ny - 1), (1, Nx - 2), 3),
                                    (VY, k3, (g.fs, Nz - 1), (1, Ny - 2), (1, Nx - 1), 2),
                                    (VZ, k4, (g.fs, Nz - 2), (1, Ny - 1), (1, Nx - 1), 1)):
        (za, zb), (ya, yb), (xa, xb) = zr, yr, xr
        if zb <= za or yb <= ya or xb <= xa:
            continue

        def sh(o):
            idx = [slice(None), slice(za, zb), slice(ya, yb), slice(xa, xb)]
            lo, hi = idx[axis].start + o, idx[axis].stop + o
            idx[axis] = slice(lo, hi)
            return pn[tuple(idx)]
        dp = d4(sh(1), sh(0), sh(2), sh(-1))
        sl = (slice(None), slice(za, zb), slice(ya, yb), slice(xa, xb))
        F[sl] = (one - k[za:zb, ya:yb, xa:xb]) * F[sl] - a2[za:zb, ya:yb, xa:xb] * dp
    if g.free_surface:
        VZ[:, g.fs - 1] = VZ[:, g.fs]
    pi = (slice(g.pml, g.pml + g.nz), slice(g.pml, g.pml + g.ny), slice(g.pml, g.pml + g.nx))
    for f in range(4):
        e = np.zeros((g.nz, g.ny, g.nx), np.float32)
        for s in range(g.S):
            v = st[s, f][pi]
            e = e + v * v
        energy[f] += e


def box(vol, z, rows, cols, g):
    """A TMA box of one plane: zero outside [0, Nz) x [0, Ny) x [0, pitch)."""
    out = np.zeros((len(rows), len(cols)), np.float32)
    if not 0 <= z < g.Nz:
        return out
    r_ok = (rows >= 0) & (rows < g.Ny)
    c_ok = (cols >= 0) & (cols < g.pitch)
    out[np.ix_(r_ok, c_ok)] = vol[z][np.ix_(rows[r_ok], cols[c_ok])]
    return out


def lanes_up(a):
    """__shfl_up_sync(v, 1): lane l gets lane l-1's value, lane 0 its own. a: (rows, 32)."""
    return np.concatenate([a[:, :1], a[:, :-1]], axis=1)


def lanes_down(a):
    return np.concatenate([a[:, 1:], a[:, -1:]], axis=1)


def cta(g, inS, outS, coef, img, src, amp, s, tx, ty, zs, ze, TY, squares, written, tma_x):
    """One CTA of step3_fused_kernel: tile (tx, ty), shot s, planes [zs, ze)."""
    a1, k1, a2, k2, k3, k4 = coef
    one = np.float32(1)
    PR, YR = TY + 3, TY + 6
    x0, y0 = tx * TX, ty * TY
    cols = x0 - 4 + np.arange(ROW)
    prow = y0 - 1 + np.arange(PR)
    vyrow = y0 - 3 + np.arange(YR)
    tma_x.add(x0 - 4)
    gx = cols.reshape(32, 4)                     # the 4 columns of each lane
    yv = prow[:, None]
    n_it = ze - zs + 3

    def stage(vol, z, rows=prow):
        return box(vol, z, rows, cols, g).reshape(len(rows), 32, 4)

    ring = np.full((4, PR, 32, 4), np.nan, np.float32)
    vzq = [np.zeros((PR, 32, 4), np.float32)] + [stage(inS[3], zs - 4 + k) for k in (1, 2, 3)]
    fs_on = g.free_surface and g.fs >= 1
    own = np.zeros((PR, 32), bool)
    own[1:TY + 1, 1:31] = True
    own &= (yv < g.Ny) & (gx[None, :, 0] < g.Nx)
    for j in range(n_it):
        zp, zv = zs - 1 + j, zs - 3 + j
        # ---- pressure of plane zp on the p rows
        vzq = vzq[1:] + [stage(inS[3], zp + 1)]
        p = stage(inS[0], zp)
        xc = stage(inS[1], zp)
        xs = [lanes_up(xc[..., 2]), lanes_up(xc[..., 3]), xc[..., 0], xc[..., 1], xc[..., 2], xc[..., 3],
              lanes_down(xc[..., 0])]
        vy = stage(inS[2], zp, vyrow)
        if g.fs + 1 <= zp < g.Nz - 2:
            A1, K1 = stage(a1, zp), stage(k1, zp)
            own_p = own & (zs <= zp < ze)
            for q in range(4):
                m = (yv >= 2) & (yv < g.Ny - 2) & (gx[None, :, q] >= 2) & (gx[None, :, q] < g.Nx - 2)
                dvx = d4(xs[q + 2], xs[q + 1], xs[q + 3], xs[q])
                dvy = d4(vy[2:2 + PR, :, q], vy[1:1 + PR, :, q], vy[3:3 + PR, :, q], vy[0:PR, :, q])
                dvz = d4(vzq[2][..., q], vzq[1][..., q], vzq[3][..., q], vzq[0][..., q])
                ssum = (dvx + dvy) + dvz
                p[..., q] = np.where(m, (one - K1[..., q]) * p[..., q] - A1[..., q] * ssum, p[..., q])
                for r, l in zip(*np.nonzero(m & own_p)):
                    img["i"][s, zp, prow[r], gx[l, q]] = -ssum[r, l]
        if zp == src[0]:
            for r in np.nonzero(prow == src[1])[0]:
                for l in range(32):
                    if gx[l, 0] <= src[2] < gx[l, 0] + 4:
                        p[r, l, src[2] - gx[l, 0]] += amp
        ring[zp & 3] = p
        if fs_on and zp == g.fs + 1:
            ring[(g.fs - 1) & 3] = -p
        if j < 3:
            continue
        # ---- velocities of plane zv on the tile
        pc = ring[zv & 3]
        ps = [lanes_up(pc[..., 3]), pc[..., 0], pc[..., 1], pc[..., 2], pc[..., 3], lanes_down(pc[..., 0]),
              lanes_down(pc[..., 1])]
        vx, vyv, vz = stage(inS[1], zv), stage(inS[2], zv), vzq[0].copy()
        A2, K2, K3, K4 = (stage(c, zv) for c in (a2, k2, k3, k4))
        zin, zinz = g.fs <= zv < g.Nz - 1, g.fs <= zv < g.Nz - 2
        for q in range(4):
            xq = gx[None, :, q]
            m = zin & (yv >= 1) & (yv < g.Ny - 1) & (xq >= 1) & (xq < g.Nx - 2)
            dp = d4(ps[q + 2], ps[q + 1], ps[q + 3], ps[q])
            vx[..., q] = np.where(m, (one - K2[..., q]) * vx[..., q] - A2[..., q] * dp, vx[..., q])
            for r, l in zip(*np.nonzero(m & own)):
                img["j"][0, s, zv, prow[r], gx[l, q]] = dp[r, l]
            m = zin & (yv >= 1) & (yv < g.Ny - 2) & (xq >= 1) & (xq < g.Nx - 1)
            col = pc[..., q]
            ym1, yp1, yp2 = np.roll(col, 1, 0), np.roll(col, -1, 0), np.roll(col, -2, 0)   # rows of the tile only
            dp = d4(yp1, col, yp2, ym1)
            vyv[..., q] = np.where(m, (one - K3[..., q]) * vyv[..., q] - A2[..., q] * dp, vyv[..., q])
            for r, l in zip(*np.nonzero(m & own)):
                img["j"][1, s, zv, prow[r], gx[l, q]] = dp[r, l]
            m = zinz & (yv >= 1) & (yv < g.Ny - 1) & (xq >= 1) & (xq < g.Nx - 1)
            dp = d4(ring[(zv + 1) & 3][..., q], col, ring[(zv + 2) & 3][..., q], ring[(zv - 1) & 3][..., q])
            vz[..., q] = np.where(m, (one - K4[..., q]) * vz[..., q] - A2[..., q] * dp, vz[..., q])
            for r, l in zip(*np.nonzero(m & own)):
                img["j"][2, s, zv, prow[r], gx[l, q]] = dp[r, l]
        squares[(zv, tx, ty, s)] = [v[1:TY + 1] * v[1:TY + 1] for v in (pc, vx, vyv, vz)]
        for r, l in zip(*np.nonzero(own)):
            y, c = prow[r], gx[l, 0]
            for f, v in enumerate((pc, vx, vyv)):
                outS[f, zv, y, c:c + 4] = v[r, l]
                written[f, zv, y, c:c + 4] += 1
            if not (fs_on and zv == g.fs - 1):
                outS[3, zv, y, c:c + 4] = vz[r, l]
                written[3, zv, y, c:c + 4] += 1
            if fs_on and zv == g.fs:
                outS[3, g.fs - 1, y, c:c + 4] = vz[r, l]
                written[3, g.fs - 1, y, c:c + 4] += 1


def fused_step(g, inb, outb, coef, img, src, amp, energy, TY, chunk, written, tma_x):
    tiles_x, tiles_y = (g.Nx + TX - 1) // TX, (g.Ny + TY - 1) // TY
    for zs in range(0, g.Nz, chunk):
        ze = min(g.Nz, zs + chunk)
        for ty in range(tiles_y):
            for tx in range(tiles_x):
                squares = {}
                for s in range(g.S):
                    cta(g, inb[s], outb[s], coef, img, src[s], amp[s], s, tx, ty, zs, ze, TY, squares, written[s],
                        tma_x)
                # the cluster of this tile: each plane's squares over the shots, in shot order
                for zv in range(max(zs, g.pml), min(ze, g.pml + g.nz)):
                    for f in range(4):
                        tot = squares[(zv, tx, ty, 0)][f]
                        for s in range(1, g.S):
                            tot = tot + squares[(zv, tx, ty, s)][f]
                        for row in range(TY):
                            y = ty * TY + row
                            if not g.pml <= y < g.pml + g.ny:
                                continue
                            for lane in range(1, 31):
                                for q in range(4):
                                    x = tx * TX - 4 + 4 * lane + q
                                    if g.pml <= x < g.pml + g.nx:
                                        e = energy[f]
                                        e[zv - g.pml, y - g.pml, x - g.pml] += tot[row, lane, q]


def split_img(g, st, coef):
    """The imaging fields p3_kernel / v3_kernel write for one step (the
    divergence on the p mask; the pressure derivatives on the velocity masks)."""
    Nz, Ny, Nx = g.Nz, g.Ny, g.Nx
    P, VX, VY, VZ = (st[:, f] for f in range(4))
    ii = np.zeros((g.S, Nz, Ny, g.pitch), np.float32)
    z0, z1, y0, y1, x0, x1 = g.fs + 1, Nz - 2, 2, Ny - 2, 2, Nx - 2
    if z1 > z0 and y1 > y0 and x1 > x0:
        sl = (slice(None), slice(z0, z1), slice(y0, y1), slice(x0, x1))
        dvx = d4(VX[sl], VX[:, z0:z1, y0:y1, x0 - 1:x1 - 1], VX[:, z0:z1, y0:y1, x0 + 1:x1 + 1],
                 VX[:, z0:z1, y0:y1, x0 - 2:x1 - 2])
        dvy = d4(VY[sl], VY[:, z0:z1, y0 - 1:y1 - 1, x0:x1], VY[:, z0:z1, y0 + 1:y1 + 1, x0:x1],
                 VY[:, z0:z1, y0 - 2:y1 - 2, x0:x1])
        dvz = d4(VZ[sl], VZ[:, z0 - 1:z1 - 1, y0:y1, x0:x1], VZ[:, z0 + 1:z1 + 1, y0:y1, x0:x1],
                 VZ[:, z0 - 2:z1 - 2, y0:y1, x0:x1])
        ii[sl] = -((dvx + dvy) + dvz)
    return ii


def split_img_j(g, pn):
    Nz, Ny, Nx = g.Nz, g.Ny, g.Nx
    jj = np.zeros((3, g.S, Nz, Ny, g.pitch), np.float32)
    for c, (zr, yr, xr, axis) in enumerate((((g.fs, Nz - 1), (1, Ny - 1), (1, Nx - 2), 3),
                                            ((g.fs, Nz - 1), (1, Ny - 2), (1, Nx - 1), 2),
                                            ((g.fs, Nz - 2), (1, Ny - 1), (1, Nx - 1), 1))):
        (za, zb), (ya, yb), (xa, xb) = zr, yr, xr

        def sh(o):
            idx = [slice(None), slice(za, zb), slice(ya, yb), slice(xa, xb)]
            idx[axis] = slice(idx[axis].start + o, idx[axis].stop + o)
            return pn[tuple(idx)]
        jj[c][:, za:zb, ya:yb, xa:xb] = d4(sh(1), sh(0), sh(2), sh(-1))
    return jj


def run_case(nz, ny, nx, pml, S, free_surface, chunk, steps=3, TY=8, seed=0):
    g = Geo(nz, ny, nx, pml, S, free_surface)
    rng = np.random.default_rng(seed)
    shp = (g.Nz, g.Ny, g.pitch)

    def vol(scale, lo=0.0):
        v = np.zeros(shp, np.float32)
        v[:, :, :g.Nx] = (lo + scale * rng.random((g.Nz, g.Ny, g.Nx))).astype(np.float32)
        return v
    coef = [vol(0.3, 0.1), vol(0.02), vol(0.3, 0.1), vol(0.02), vol(0.02), vol(0.02)]
    # sources: one on the grid's edge, one in a tile's halo column, the rest at random
    src = [(1, 0, 0), (min(g.fs + 1, g.Nz - 1), g.Ny // 2, min(TX - 1, g.Nx - 1))]
    src += [tuple(int(rng.integers(0, n)) for n in (g.Nz, g.Ny, g.Nx)) for _ in range(S)]
    src = src[:S]
    st = np.zeros((S, 4) + shp, np.float32)
    st[..., :g.Nx] = (rng.standard_normal((S, 4, g.Nz, g.Ny, g.Nx)) * 0.1).astype(np.float32)
    ref, cur = st.copy(), st.copy()
    other = np.full_like(st, np.nan)
    c4 = (g.Nx + 3) // 4 * 4
    other[..., c4:] = 0.0                    # never written: zero since the buffers were cleared
    e_ref = [np.zeros((nz, ny, nx), np.float32) for _ in range(4)]
    e_fus = [np.zeros((nz, ny, nx), np.float32) for _ in range(4)]
    tma_x = set()
    for it in range(steps):
        amp = rng.standard_normal(S).astype(np.float32)
        ii = split_img(g, ref, coef)
        split_step(g, ref, coef, src, amp, e_ref)
        jj = split_img_j(g, ref[:, 0])
        img = {"i": np.zeros_like(ii), "j": np.zeros_like(jj)}
        written = np.zeros((S, 4) + shp, np.int32)
        fused_step(g, cur, other, coef, img, src, amp, e_fus, TY, chunk, written, tma_x)
        assert (written[..., :c4] == 1).all(), "every cell written exactly once"
        assert (written[..., c4:] == 0).all()
        np.testing.assert_array_equal(other, ref)
        np.testing.assert_array_equal(img["i"], ii)
        np.testing.assert_array_equal(img["j"], jj)
        cur, other = other, cur
    for f in range(4):
        np.testing.assert_array_equal(e_fus[f], e_ref[f])
    assert all(x % 4 == 0 for x in tma_x)


@pytest.mark.parametrize("free_surface", [False, True])
@pytest.mark.parametrize("nz,ny,nx,pml,S,chunk", [
    (12, 10, 14, 3, 2, 100),   # one chunk
    (12, 10, 14, 3, 2, 5),     # chunks of 5 planes: the mirror planes across a chunk edge
    (9, 13, 117, 2, 3, 4),     # two x tiles (Nx = 121), a ragged last float4, ragged y tiles
    (6, 5, 7, 2, 1, 3),        # tiny grid, one shot
])
def test_fused_dataflow_equals_split_step(nz, ny, nx, pml, S, free_surface, chunk):
    run_case(nz, ny, nx, pml, S, free_surface, chunk)


@pytest.mark.parametrize("free_surface", [False, True])
def test_fused_dataflow_with_16_row_tiles(free_surface):
    run_case(12, 25, 14, 3, 2, free_surface, 5, TY=16)


def test_chunk_choice_fills_waves():
    """f3_chunks (gb_capi3d.cu) restated: the chosen chunk count for the
    200^3 + 20 PML, 4-shot workload (60 tiles of 8 x 120) on 148 SMs x 2."""
    def chunks(Nz, tiles, ns, slots):
        best, best_eff = 1, 0.0
        for c in range(1, 33):
            chunk = (Nz + c - 1) // c
            if chunk < 4 and c > 1:
                break
            n = (Nz + chunk - 1) // chunk
            work = n * tiles * ns
            waves = (work + slots - 1) // slots
            eff = work / (waves * slots) * chunk / (chunk + 3.0)
            if eff > best_eff + 1e-9:
                best, best_eff = n, eff
        return best, best_eff
    n, eff = chunks(240, 2 * 30, 4, 296)
    assert n == 6 and eff > 0.9
