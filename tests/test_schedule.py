"""The CTA work lists of schedule mode 1 (gb_plan_set_schedule), read
through gb_plan_schedule_items on the host (plan creation and the list
builder make no device call; positions are unpadded, as the reference
takes them).  Every (tile, shot) pair of a launch appears in exactly one
item, an item's shots lie in one shot group, the tiles that take the slow
path come first, only the last items (one per resident slot) are split,
and the lists fit the workspace region the layout sets aside for them."""
import ctypes

import numpy as np
import pytest

from test_capi import lib  # noqa: F401  (module fixture: the built library)

TX = 120


def _plan(lib, nz, nx, nabc, half, n_shots, free_surface=0):
    from geobrain_b200 import _lib
    d = _lib.ModelDesc(nz=nz, nx=nx, nabc=nabc, nt=10, n_shots=n_shots, n_rcv=nx, half=half,
                       free_surface=free_surface, dt=1e-3, dx=10.0)
    sx = np.linspace(0, nx - 1, n_shots).astype(np.int64)
    sz = np.ones(n_shots, np.int64)
    rx = np.arange(nx, dtype=np.int64)
    rz = np.ones(nx, np.int64)
    h = ctypes.c_void_p()
    assert lib.gb_plan_create(ctypes.byref(d), sx.ctypes.data, sz.ctypes.data, rx.ctypes.data, rz.ctypes.data,
                              ctypes.byref(h)) == 0, lib.gb_last_error()
    return h


def _items(lib, h, slots, config):
    n = ctypes.c_int()
    assert lib.gb_plan_schedule_items(h, slots, config, None, 0, ctypes.byref(n)) == 0, lib.gb_last_error()
    buf = np.zeros(3 * max(n.value, 1), np.int32)
    assert lib.gb_plan_schedule_items(h, slots, config, buf.ctypes.data, n.value, ctypes.byref(n)) == 0
    return buf[:3 * n.value].reshape(-1, 3)


@pytest.mark.parametrize("nz,nx,nabc,half,shots,free_surface,spc", [
    (400, 1200, 30, 4, 32, 0, 0),   # the 400 x 1200, 32-shot workload: 8 shots per CTA, 4 groups
    (60, 250, 10, 4, 7, 0, 2),      # groups of 2, 2, 2, 1
    (100, 200, 20, 2, 5, 1, 3),     # free surface, 4th order
    (37, 53, 4, 2, 1, 0, 0),        # one tile row, one shot
])
@pytest.mark.parametrize("slots", [1, 5, 37, 296])
def test_work_lists_cover_every_tile_and_shot_once(lib, nz, nx, nabc, half, shots, free_surface, spc, slots):
    h = _plan(lib, nz, nx, nabc, half, shots, free_surface)
    try:
        assert lib.gb_plan_set_tiling(h, 16, spc) == 0, lib.gb_last_error()
        tz, spc_eff, streams, gsteps, chunks, rrows = (ctypes.c_int() for _ in range(6))
        assert lib.gb_plan_get_config(h, *(ctypes.byref(v) for v in (tz, spc_eff, streams, gsteps, chunks,
                                                                     rrows))) == 0
        spc_eff = spc_eff.value
        n_groups = -(-shots // spc_eff)
        Nz, Nx = nz + 2 * nabc, nx + 2 * nabc
        tiles_x, tiles_z = -(-Nx // TX), -(-Nz // 16)
        n_tiles = tiles_x * tiles_z
        R = half
        fs = nabc if free_surface else 1
        zlo, zhi, xlo, xhi = max(fs + 1, nabc), nabc + nz, nabc, nabc + nx

        def slow(t):
            z0, x0 = (t // tiles_x) * 16, (t % tiles_x) * TX
            return not (z0 - 2 * R >= zlo and z0 + 16 + 2 * R <= zhi and x0 - 8 >= xlo and x0 + TX + 8 <= xhi)

        total = 0
        for config in range(n_groups + 1):
            it = _items(lib, h, slots, config)
            total += len(it)
            groups = [config] if config < n_groups else list(range(n_groups))
            want = {(t, s) for t in range(n_tiles) for g in groups
                    for s in range(g * spc_eff, min(shots, (g + 1) * spc_eff))}
            seen = []
            for t, s0, ns in it:
                assert 0 <= t < n_tiles and ns >= 1 and ns <= 64
                assert s0 // spc_eff == (s0 + ns - 1) // spc_eff, "an item within one shot group"
                seen += [(int(t), s) for s in range(s0, s0 + ns)]
            assert len(seen) == len(set(seen)) and set(seen) == want
            # tiles in order of first appearance: the slow-path ones first
            order = list(dict.fromkeys(int(t) for t in it[:, 0]))
            flags = [slow(t) for t in order]
            assert flags == sorted(flags, reverse=True)
            # the list is the (tile, group) items in that tile order, with the
            # last ones (one per resident slot of the launch) split into halves
            concurrent = n_groups if n_groups > 1 else 1
            per_launch = max(1, slots // concurrent) if config < n_groups else slots
            base = [(t, g * spc_eff, min(shots, (g + 1) * spc_eff) - g * spc_eff) for t in order for g in groups]
            first_split = max(0, len(base) - per_launch)
            expect = list(base[:first_split])
            for t, s0, ns in base[first_split:]:
                expect += [(t, s0, ns // 2), (t, s0 + ns // 2, ns - ns // 2)] if ns >= 2 else [(t, s0, ns)]
            assert [tuple(int(v) for v in row) for row in it] == expect
        assert total <= 4 * n_tiles * max(n_groups, 1)
    finally:
        lib.gb_plan_destroy(h)


def test_schedule_items_refuses_bad_arguments(lib):
    from geobrain_b200 import _lib
    h = _plan(lib, 60, 250, 10, 4, 7)
    try:
        n = ctypes.c_int()
        for slots, config in ((0, 0), (296, -1), (296, 99)):
            assert lib.gb_plan_schedule_items(h, slots, config, None, 0, ctypes.byref(n)) == _lib.GB_E_ARG
        assert lib.gb_plan_schedule_items(h, 296, 0, None, 0, ctypes.byref(n)) == 0 and n.value > 0
        buf = np.zeros(3, np.int32)
        if n.value > 1:
            assert lib.gb_plan_schedule_items(h, 296, 0, buf.ctypes.data, 1, ctypes.byref(n)) == _lib.GB_E_ARG
        assert lib.gb_plan_set_schedule(h, 2) == _lib.GB_E_ARG
    finally:
        lib.gb_plan_destroy(h)
