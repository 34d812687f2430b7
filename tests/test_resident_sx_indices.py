"""CPU check of the one-exchange-a-step resident kernel's index arithmetic
(gb_resident_sx.cuh: sx_send, sx_halo and the p / v item loops, restated):
every halo group a tile polls for is sent by the right neighbour into the
same words, with the cells the receiver expects; no word is sent twice in a
step; every index stays inside its strip slot and shared-memory rect.  A
group polled for but never sent would leave the receiver polling until its
bound."""
import pytest

R, H, TX = 2, 4, 120          # 4th order; halo rows 2R; tile columns
N_DIRS = 8                    # up, down, left, right, up-left, up-right, down-left, down-right


def neighbours(t, tiles_x, tiles_z):
    ti, tj = divmod(t, tiles_x)
    up, dn, lf, rt = ti > 0, ti + 1 < tiles_z, tj > 0, tj + 1 < tiles_x
    return [t - tiles_x if up else -1, t + tiles_x if dn else -1,
            t - 1 if lf else -1, t + 1 if rt else -1,
            t - tiles_x - 1 if up and lf else -1, t - tiles_x + 1 if up and rt else -1,
            t + tiles_x - 1 if dn and lf else -1, t + tiles_x + 1 if dn and rt else -1]


def check(Nz, Nx, TZ):
    tiles_x, tiles_z = (Nx + TX - 1) // TX, (Nz + TZ - 1) // TZ
    rows, prows = TZ + 2 * H, TZ + 2 * R
    band = H * 30
    groups = max(band, TZ)
    slot = N_DIRS * 2 * groups * 4
    seg = 2 * band + 2 * TZ + 4 * H

    def word(d, f, g):
        return ((d * 2 + f) * groups + g) * 4

    sent = {}                 # (tile, word) -> (global row, global column of the 4 cells, field)
    for t in range(tiles_x * tiles_z):
        ti, tj = divmod(t, tiles_x)
        z0, x0 = ti * TZ, tj * TX
        nb = neighbours(t, tiles_x, tiles_z)
        for i in range(TZ * 30):
            r, l = H + i // 30, 1 + i % 30
            top, bot = r < 2 * H, r >= TZ

            def put(d, g):
                if nb[d] < 0:
                    return
                assert 0 <= g < groups, (d, g)
                for f in (0, 1):
                    w = word(d, f, g)
                    assert 0 <= w and w + 3 < slot
                    assert (t, w) not in sent, ("two sends to one word", t, w)
                    sent[(t, w)] = (z0 - H + r, x0 - 4 + 4 * l, f)

            if top:
                put(0, (r - H) * 30 + l - 1)
            if bot:
                put(1, (r - TZ) * 30 + l - 1)
            if l == 1:
                put(2, r - H)
                if top:
                    put(4, r - H)
                if bot:
                    put(6, r - TZ)
            if l == 30:
                put(3, r - H)
                if top:
                    put(5, r - H)
                if bot:
                    put(7, r - TZ)

    received = 0
    for t in range(tiles_x * tiles_z):
        ti, tj = divmod(t, tiles_x)
        z0, x0 = ti * TZ, tj * TX
        nb = neighbours(t, tiles_x, tiles_z)
        dsts = set()
        for h in range(2 * seg):
            f, k = divmod(h, seg)
            if k < band:
                d, sd, j = 0, 1, k
                row, col = j // 30, 4 * (1 + j % 30)
            elif k < 2 * band:
                d, sd, j = 1, 0, k - band
                row, col = TZ + H + j // 30, 4 * (1 + j % 30)
            elif k < 2 * band + TZ:
                d, sd, j = 2, 3, k - 2 * band
                row, col = H + j, 0
            elif k < 2 * band + 2 * TZ:
                d, sd, j = 3, 2, k - 2 * band - TZ
                row, col = H + j, 124
            else:
                c = k - 2 * band - 2 * TZ
                j, d = c % H, 4 + c // H
                sd = 11 - d
                row = j if d < 6 else TZ + H + j
                col = 124 if d & 1 else 0
            assert 0 <= row < rows and 0 <= col <= 124
            assert (f, row, col) not in dsts
            dsts.add((f, row, col))
            if nb[d] < 0:
                continue
            w = word(sd, f, j)
            assert 0 <= w and w + 3 < slot
            assert (nb[d], w) in sent, ("received but never sent", t, d, sd, j, f)
            assert sent[(nb[d], w)] == (z0 - H + row, x0 - 4 + col, f), ("wrong cells", t, d, j, f)
            received += 1

    # the p items (lanes 1..30) and the edge cells (columns 3, 124, 125) read
    # vx and vz inside the rect; the v items read p rows the p update wrote
    for i in range(prows * 30):
        r = R + i // 30
        assert 0 <= r - R and r + R - 1 < rows
    for j in range(3 * prows):
        r, k = R + j // 3, j % 3
        c = 3 if k == 0 else 123 + k
        assert r - R >= 0 and r + R - 1 < rows and c - R >= 1 and c + R - 1 <= 127
    for i in range(TZ * 30):
        r = H + i // 30
        assert r - R + 1 >= R and r + R < R + prows
    return len(sent), received


@pytest.mark.parametrize("Nz,Nx", [(140, 240), (45, 61), (80, 270), (170, 350)])
@pytest.mark.parametrize("TZ", [4, 8, 12, 16, 24, 32, 36, 40])
def test_every_received_group_is_sent(Nz, Nx, TZ):
    if (Nx + TX - 1) // TX * ((Nz + TZ - 1) // TZ) > 148:
        pytest.skip("more tiles than SMs: the plan does not choose this tiling")
    sent, received = check(Nz, Nx, TZ)
    assert received > 0 or (Nx <= TX and Nz <= TZ)
