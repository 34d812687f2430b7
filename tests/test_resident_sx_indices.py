"""CPU check of the one-exchange-a-step resident kernel's index arithmetic
(gb_resident_sx.cuh: sx_send, sx_halo and the p / v item loops, restated):
every halo group a tile polls for is sent by the right neighbour into the
same words, with the cells the receiver expects; no word is sent twice in a
step; every index stays inside its strip slot and shared-memory rect.  A
group polled for but never sent would leave the receiver polling until its
bound."""
import pytest

R, H, RS = 2, 4, 132
def check(Nz, Nx, TZ, NW):
    TX = 120
    tiles_x = (Nx + TX - 1) // TX; tiles_z = (Nz + TZ - 1) // TZ
    ROWS = TZ + 2 * H; PROWS = TZ + 2 * R; BAND = H * 30; GROUPS = max(BAND, TZ)
    SLOT = 8 * 2 * GROUPS * 4; SEG = 2 * BAND + 2 * TZ + 4 * H; NRECV = 2 * SEG
    word = lambda d, f, g: ((d * 2 + f) * GROUPS + g) * 4
    def nbs(t):
        ti, tj = divmod(t, tiles_x)
        up, dn, lf, rt = ti > 0, ti + 1 < tiles_z, tj > 0, tj + 1 < tiles_x
        return [t - tiles_x if up else -1, t + tiles_x if dn else -1, t - 1 if lf else -1, t + 1 if rt else -1,
                t - tiles_x - 1 if up and lf else -1, t - tiles_x + 1 if up and rt else -1,
                t + tiles_x - 1 if dn and lf else -1, t + tiles_x + 1 if dn and rt else -1]
    sent = {}   # (tile, word) -> (global z, global x0 of the 4 cells, field)
    for t in range(tiles_x * tiles_z):
        ti, tj = divmod(t, tiles_x); z0, x0 = ti * TZ, tj * TX; nb = nbs(t)
        for i in range(TZ * 30):
            r, l = H + i // 30, 1 + i % 30
            assert H <= r < H + TZ
            top, bot = r < 2 * H, r >= TZ
            def put(d, g):
                if nb[d] < 0: return
                assert 0 <= g < GROUPS, (d, g)
                for f in (0, 1):
                    w = word(d, f, g); assert 0 <= w and w + 3 < SLOT
                    key = (t, w)
                    assert key not in sent, ("two sends to one word", key)
                    sent[key] = (z0 - H + r, x0 - 4 + 4 * l, f)
            if top: put(0, (r - H) * 30 + l - 1)
            if bot: put(1, (r - TZ) * 30 + l - 1)
            if l == 1:
                put(2, r - H)
                if top: put(4, r - H)
                if bot: put(6, r - TZ)
            if l == 30:
                put(3, r - H)
                if top: put(5, r - H)
                if bot: put(7, r - TZ)
    nrecv = 0
    for t in range(tiles_x * tiles_z):
        ti, tj = divmod(t, tiles_x); z0, x0 = ti * TZ, tj * TX; nb = nbs(t)
        dsts = set()
        for h in range(NRECV):
            f, k = divmod(h, SEG)
            if k < BAND: d, sd, j = 0, 1, k; row, col = j // 30, 4 * (1 + j % 30)
            elif k < 2 * BAND: d, sd, j = 1, 0, k - BAND; row, col = TZ + H + j // 30, 4 * (1 + j % 30)
            elif k < 2 * BAND + TZ: d, sd, j = 2, 3, k - 2 * BAND; row, col = H + j, 0
            elif k < 2 * BAND + 2 * TZ: d, sd, j = 3, 2, k - 2 * BAND - TZ; row, col = H + j, 124
            else:
                c = k - 2 * BAND - 2 * TZ; j = c % H; d = 4 + c // H; sd = 11 - d
                row = j if d < 6 else TZ + H + j; col = 124 if d & 1 else 0
            assert 0 <= row < ROWS and 0 <= col <= 124
            assert (f, row, col) not in dsts; dsts.add((f, row, col))
            if nb[d] < 0: continue
            w = word(sd, f, j); assert 0 <= w and w + 3 < SLOT
            key = (nb[d], w)
            assert key in sent, ("received but never sent", t, d, sd, j, f)
            gz, gx, ff = sent[key]
            assert (gz, gx, ff) == (z0 - H + row, x0 - 4 + col, f), ("wrong cells", t, d, key, sent[key], (z0 - H + row, x0 - 4 + col, f))
            nrecv += 1
        # every halo cell the stencils read is received or off the grid / filled at launch start
    # p items and edge cells
    for i in range(PROWS * 30 + 3 * PROWS):
        if i < PROWS * 30:
            r, l = R + i // 30, 1 + i % 30
            assert 0 <= r - R and r + R - 1 < ROWS and 0 <= r - R < PROWS
        else:
            j = i - PROWS * 30; r, k = R + j // 3, j % 3; c = 3 if k == 0 else 123 + k
            assert 0 <= r - 1 - (R - 1) and r + R - 1 < ROWS and 1 <= c - R and c + R - 1 <= 127
    for i in range(TZ * 30):
        r = H + i // 30
        assert r - R + 1 >= R and r + R < R + PROWS      # p rows read by the v update are updated rows
    return len(sent), nrecv


@pytest.mark.parametrize("Nz,Nx", [(140, 240), (45, 61), (80, 270), (170, 350)])
@pytest.mark.parametrize("TZ,NW", [(4, 8), (8, 8), (12, 8), (16, 8), (24, 16), (32, 16), (36, 16), (40, 16)])
def test_every_received_group_is_sent(Nz, Nx, TZ, NW):
    if (Nx + 119) // 120 * ((Nz + TZ - 1) // TZ) > 148:
        pytest.skip("more tiles than SMs: the plan does not choose this tiling")
    sent, received = check(Nz, Nx, TZ, NW)
    assert received > 0 or (Nx <= 120 and Nz <= TZ)
