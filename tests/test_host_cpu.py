"""CPU tests: case builder, reference file formats, host set-up code against
the reference's own set-up, and the C-ABI library's exported symbols."""
import json
import os
import re
import tempfile

import numpy as np
import pytest

import refio
from orion_b200 import cases, solver
from parity import ROOT

HEADER = os.path.join(ROOT, "include", "orion_gpu.h")
needs_ref = pytest.mark.skipif(not refio.reference_available(), reason="oracle/_ref not built")


def header_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(orion_[a-z_0-9]+)\s*\(", txt, flags=re.M)))


def test_library_exports_every_header_symbol():
    from orion_b200 import _lib

    lib = _lib.load()
    names = header_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(_lib.SIGNATURES), set(names) ^ set(_lib.SIGNATURES)
    assert lib.orion_abi_version() == 1


def test_library_rejects_bad_arguments_without_gpu():
    import ctypes as C

    from orion_b200 import _lib

    lib = _lib.load()
    h = C.c_void_p()
    # nblocks <= 0 is rejected before any device work
    rc = lib.orion_case_create(0, None, C.byref(_lib.Params()), 0, C.byref(h))
    assert rc == -1
    assert b"nblocks" in lib.orion_last_error()
    assert lib.orion_exchange_bc(None) == -1


def test_split_topology_is_consistent():
    c = cases.small_case("t", dims=(33, 25, 23), split=(2, 2, 2))
    assert len(c.blocks) == 8
    for n, b in enumerate(c.blocks):
        assert len(b.regions) == 6
        for r, g in enumerate(b.regions):
            if g.bctype < 0:
                partner = c.blocks[g.nbt - 1].regions[g.ibcwin - 1]
                assert partner.bctype < 0
                assert partner.nbt == n + 1 and partner.ibcwin == r + 1
                # point-matched windows of equal extent
                ext_s = [abs(g.s_ed[d] - g.s_st[d]) for d in range(3)]
                ext_t = [abs(partner.s_ed[d] - partner.s_st[d]) for d in range(3)]
                assert ext_s == ext_t
                # shared plane: coordinates coincide
                b2 = c.blocks[g.nbt - 1]
                d = g.normal_dir() - 1
                sl_a = [slice(None)] * 3
                sl_b = [slice(None)] * 3
                sl_a[2 - d] = g.s_st[d] - 1
                sl_b[2 - d] = partner.s_st[d] - 1
                assert np.array_equal(b.x[tuple(sl_a)], b2.x[tuple(sl_b)])
                assert np.array_equal(b.y[tuple(sl_a)], b2.y[tuple(sl_b)])


def test_uneven_split_ratio_and_minimum():
    c = cases.config(2)
    ext = {}
    for b in c.blocks:
        for d, v in enumerate(b.dims):
            ext.setdefault(d, []).append(v - 1)
    for d, v in ext.items():
        assert min(v) >= cases.MIN_BLOCK_DIM - 1
        assert max(v) <= 3 * min(v) + 1
    assert sum(b.npoints for b in c.blocks) > 289 * 161 * 65


def test_noise_stream_matches_scalar_splitmix():
    def scalar(seed, k):
        mask = (1 << 64) - 1
        z = (seed + k * 0x9E3779B97F4A7C15) & mask
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & mask
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & mask
        z = z ^ (z >> 31)
        return (z >> 11) * (1.0 / 9007199254740992.0)

    v = cases.splitmix64_uniform(123, 5, 4)
    assert list(v) == [scalar(123, k) for k in range(6, 10)]


def test_reference_file_formats_roundtrip(tmp_path):
    c = cases.small_case("fmt", dims=(17, 13, 12), split=(1, 1, 1))
    c.write_reference_inputs(str(tmp_path))
    raw = open(tmp_path / "grid.x", "rb").read()
    n = np.frombuffer(raw, dtype="<u4", count=1)[0]
    assert n == 4 and np.frombuffer(raw, dtype="<i4", count=1, offset=4)[0] == 1
    lines = open(tmp_path / "bc.inp").read().split("\n")
    assert lines[0] == "1976" and lines[2] == "1"
    txt = open(tmp_path / "param.dat").read()
    assert "$inflow" in txt and "gcl = 1" in txt


@needs_ref
@pytest.mark.parametrize("split", [(1, 1, 1), (2, 2, 2)])
def test_host_metrics_and_init_match_reference_setup(split, tmp_path):
    """orion_grid_metrics_host and the seeded initial state are bit-identical to
    compute_grid_metrics/check_grid_metrics and initialize_flow/update_temperature."""
    c = cases.small_case("m", dims=(29, 25, 23), split=split, nsteps=0, noise_seed=3)
    c.write_reference_inputs(str(tmp_path / "case"))
    refio.run_reference(str(tmp_path / "case"), 0, str(tmp_path / "out"))
    ref = refio.read_state(str(tmp_path / "out" / "init.bin"))
    prims = solver.initial_prim(c)
    for n, b in enumerate(c.blocks):
        met, vol = solver.grid_metrics(b, 1)
        assert np.array_equal(met, ref["blocks"][n]["metrics"])
        assert np.array_equal(vol, ref["blocks"][n]["vol"])
        assert np.array_equal(prims[n], ref["blocks"][n]["prim"])


def test_metrics_unit_cube_volume():
    """Unit-cube known answer (orion_bench test 2, src/benchmark.cpp:109-165):
    x=i, y=j, z=k gives vol == 1 at every interior point."""
    n = 14
    k, j, i = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    blk = cases.Block(n, n, n, i.astype(float), j.astype(float), k.astype(float))
    for gcl in (0, 1):
        met, vol = solver.grid_metrics(blk, gcl)
        assert np.max(np.abs(vol[3:-3, 3:-3, 3:-3] - 1.0)) < 1e-12
        assert np.all(vol[:3] == 0)


@needs_ref
@pytest.mark.parametrize("key", ["small_1blk", "small_8blk", "small_bcmix", "small_euler"])
def test_golden_fixtures_reproduce(key, tmp_path):
    """The committed golden fixtures are what the reference produces today."""
    import sys

    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import gen_golden

    case = gen_golden.build(gen_golden.RECIPES[key])
    case.write_reference_inputs(str(tmp_path / "case"))
    refio.run_reference(str(tmp_path / "case"), case.nsteps, str(tmp_path / "out"))
    g = np.load(os.path.join(ROOT, "tests", "golden", key + ".npz"))
    hist = refio.read_hist(str(tmp_path / "out" / "hist.bin"))
    final = refio.read_state(str(tmp_path / "out" / "final.bin"))
    assert np.array_equal(hist, g["hist"])
    assert np.array_equal(gen_golden.interior_prim(final, int(g["sub"][0])), g["prim"])


def test_golden_fixture_recipes_load():
    for f in ("small_1blk", "small_8blk", "small_uneven", "small_bcmix", "small_euler"):
        g = np.load(os.path.join(ROOT, "tests", "golden", f + ".npz"))
        recipe = json.loads(str(g["recipe"][0]))
        c = cases.small_case(**recipe)
        assert g["hist"].shape == (c.nsteps, 8)
        assert np.all(np.isfinite(g["hist"]))
