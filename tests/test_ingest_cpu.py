"""Case ingestion from the reference's own input formats (CPU).

read_case reads param.dat (Fortran namelist), the multi-block Plot3D grid and
the marker-1976 BC file.  A case written by write_reference_inputs reads back
identically (coordinates, signed region windows, parameters, noise), and the
reference's example inputs under testcases/NS parse (when present).
"""
import os

import numpy as np
import pytest

import refio
from orion_b200 import cases

REF_NS = os.path.join(refio.REF_ROOT, "testcases", "NS")


@pytest.mark.parametrize("split,seed", [((1, 1, 1), None), ((3, 2, 2), 4)])
def test_written_case_reads_back(tmp_path, split, seed):
    c = cases.bump_case("rt", 41, 27, 25, split=split, uneven_seed=seed, moo=0.8, reynolds=1e5, height=0.08,
                        nsteps=7, noise_seed=9)
    c.write_reference_inputs(str(tmp_path))
    r = cases.read_case(str(tmp_path))
    assert (r.nsteps, r.noise_seed, r.noise_amp) == (7, 9, c.noise_amp)
    assert r.params == c.params
    for a, b in zip(r.blocks, c.blocks):
        assert a.dims == b.dims and a.regions == b.regions
        assert np.array_equal(a.x, b.x) and np.array_equal(a.y, b.y) and np.array_equal(a.z, b.z)


def test_other_bc_types_and_flow_options_read_back(tmp_path):
    """Freestream / extrapolation faces, isothermal walls, attack, Euler and
    method 0 survive the reference's file formats."""
    c = cases.small_case("opts", dims=(33, 25, 23), split=(2, 1, 1), nsteps=4, noise_seed=3, twall=300.0,
                         attack=3.0, nvis=0, method=0,
                         physical={"imin": cases.BC_FREESTREAM, "imax": cases.BC_EXTRAPOLATION})
    types = {r.bctype for b in c.blocks for r in b.regions}
    assert {cases.BC_FREESTREAM, cases.BC_EXTRAPOLATION, cases.BC_WALL, cases.BC_INTERFACE} <= types
    c.write_reference_inputs(str(tmp_path))
    r = cases.read_case(str(tmp_path))
    assert r.params == c.params
    assert (r.params.nvis, r.params.method, r.params.twall, r.params.attack) == (0, 0, 300.0, 3.0)
    for a, b in zip(r.blocks, c.blocks):
        assert a.regions == b.regions


def test_unsupported_and_malformed_inputs_are_rejected(tmp_path):
    c = cases.small_case("bad", dims=(25, 17, 13))
    c.write_reference_inputs(str(tmp_path))
    txt = open(tmp_path / "param.dat").read().replace("height = -1.0", "height = 11.0")
    open(tmp_path / "hp.dat", "w").write(txt)
    with pytest.raises(ValueError):
        cases.read_param_dat(str(tmp_path / "hp.dat"))
    blocks = cases.read_plot3d(str(tmp_path / "grid.x"))
    blocks[0].idim += 1
    with pytest.raises(ValueError):
        cases.read_bc_inp(str(tmp_path / "bc.inp"), blocks)


@pytest.mark.skipif(not os.path.isdir(REF_NS), reason="reference example inputs not present")
def test_reference_example_inputs_parse():
    p, nomax = cases.read_param_dat(os.path.join(REF_NS, "param.dat"))
    assert (p.moo, p.reynolds, p.cfl, nomax) == (6.0, 3755.0, 1.0, 50)
    inp = os.path.join(REF_NS, "grid_64proc_out.inp")
    lines = [ln.split() for ln in open(inp) if ln.strip()]
    nb = int(lines[2][0])
    dims, pos = [], 3
    for _ in range(nb):  # walk the file once to learn the block dims (the grid itself is not shipped)
        dims.append(tuple(int(v) for v in lines[pos + 1]))
        nreg = int(lines[pos + 3][0])
        pos += 4
        for _ in range(nreg):
            pos += 2 if int(lines[pos][6]) < 0 else 1
    blocks = [cases.Block(*d, None, None, None, []) for d in dims]
    cases.read_bc_inp(inp, blocks)
    assert len(blocks) == 64 and all(len(b.regions) == 6 for b in blocks)
    iface = [r for b in blocks for r in b.regions if r.bctype < 0]
    assert iface and all(1 <= r.nbt <= 64 and r.ibcwin >= 1 for r in iface)
    assert any(min(r.s_st + r.s_ed) < 0 for r in iface)  # signed windows are kept
