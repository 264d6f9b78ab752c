"""Solution output and restart for device-resident cases.

write_solution writes what the reference's PostProcess::write_solution writes
(src/postprocess/PostProcess.cpp:43-276), byte for byte in layout:
* one VTK XML StructuredGrid file per block, `<stem>_<step:06d>_block_<nb>.vts`,
  appended raw little-endian Float32 with a UInt32 byte count before each array
  (points, Density, Pressure, Temperature, Mach, Velocity);
* a `<stem>_<step:06d>.vtm` multiblock index beside them.
The output directory and stem come from the flowname path the way the reference
splits params.filename.flowname (default "output/flow").

The fields are packed on the device (orion_case_pack_output: FP32 density,
pressure, temperature, Mach formed in FP64, velocity); write_solution_async
takes that snapshot at once and writes the files on a background thread while
the case keeps stepping.

save_restart / load_restart keep a case's state between runs: the primitive
variables of every block are the whole state between steps (every other field
is recomputed from them at the start of a step).  The reference reads nstart
but never restarts (src/preprocess/InitialCondition.cpp:10-18).
"""
from __future__ import annotations

import concurrent.futures as cf
import ctypes as C
import os
from typing import List, Optional

import numpy as np

from . import _lib
from ._lib import check

_writer = cf.ThreadPoolExecutor(max_workers=2)


def pack_block(fs, block: int) -> np.ndarray:
    """(7, n) float32: density, pressure, temperature, Mach, u, v, w at the interior points."""
    b = fs.case.blocks[block]
    n = b.idim * b.jdim * b.kdim
    out = np.empty((7, n), dtype=np.float32)
    check(_lib.load().orion_case_pack_output(fs.handle, block, out.ctypes.data))
    return out


def _split_flowname(flowname: Optional[str]):
    path = flowname or "output/flow"
    out_dir = os.path.dirname(path) or "."
    return out_dir, os.path.basename(path)


def _vts_bytes(dims, xyz: np.ndarray, f: np.ndarray) -> bytes:
    ni, nj, nk = dims
    n = ni * nj * nk
    sizes = [3 * n, n, n, n, n, 3 * n]
    offs, cur = [], 0
    for s in sizes:
        offs.append(cur)
        cur += 4 + 4 * s
    ei, ej, ek = ni - 1, nj - 1, nk - 1
    head = (
        '<?xml version="1.0"?>\n'
        '<VTKFile type="StructuredGrid" version="0.1" byte_order="LittleEndian" header_type="UInt32">\n'
        f'  <StructuredGrid WholeExtent="0 {ei} 0 {ej} 0 {ek}">\n'
        f'    <Piece Extent="0 {ei} 0 {ej} 0 {ek}">\n'
        '      <Points>\n'
        f'        <DataArray type="Float32" NumberOfComponents="3" format="appended" offset="{offs[0]}"/>\n'
        '      </Points>\n'
        '      <PointData Scalars="Density" Vectors="Velocity">\n'
        f'        <DataArray type="Float32" Name="Density" format="appended" offset="{offs[1]}"/>\n'
        f'        <DataArray type="Float32" Name="Pressure" format="appended" offset="{offs[2]}"/>\n'
        f'        <DataArray type="Float32" Name="Temperature" format="appended" offset="{offs[3]}"/>\n'
        f'        <DataArray type="Float32" Name="Mach" format="appended" offset="{offs[4]}"/>\n'
        f'        <DataArray type="Float32" Name="Velocity" NumberOfComponents="3" format="appended" offset="{offs[5]}"/>\n'
        '      </PointData>\n'
        '    </Piece>\n'
        '  </StructuredGrid>\n'
        '  <AppendedData encoding="raw">\n'
        '    _'
    ).encode()
    vel = np.stack([f[4], f[5], f[6]], axis=1).astype("<f4").ravel()
    arrays = [xyz.astype("<f4").ravel(), f[0].astype("<f4"), f[1].astype("<f4"), f[2].astype("<f4"),
              f[3].astype("<f4"), vel]
    body = b"".join(np.uint32(a.nbytes).astype("<u4").tobytes() + a.tobytes() for a in arrays)
    return head + body + b"\n  </AppendedData>\n</VTKFile>\n"


def _vtm_bytes(stem: str, step: int, nblocks: int) -> bytes:
    lines = ['<?xml version="1.0"?>\n',
             '<VTKFile type="vtkMultiBlockDataSet" version="1.0" byte_order="LittleEndian">\n',
             '  <vtkMultiBlockDataSet>\n']
    for nb in range(nblocks):
        lines.append(f'    <DataSet index="{nb}" file="{stem}_{step:06d}_block_{nb}.vts"/>\n')
    lines += ['  </vtkMultiBlockDataSet>\n', '</VTKFile>\n']
    return "".join(lines).encode()


def _snapshot(fs):
    snap = []
    for nb, b in enumerate(fs.case.blocks):
        xyz = np.stack([np.asarray(b.x, np.float64).ravel(), np.asarray(b.y, np.float64).ravel(),
                        np.asarray(b.z, np.float64).ravel()], axis=1).astype(np.float32)
        snap.append((b.dims, xyz, pack_block(fs, nb)))
    return snap


def _write(snap, flowname: Optional[str], step: int) -> List[str]:
    out_dir, stem = _split_flowname(flowname)
    os.makedirs(out_dir, exist_ok=True)
    paths = []
    for nb, (dims, xyz, f) in enumerate(snap):
        p = os.path.join(out_dir, f"{stem}_{step:06d}_block_{nb}.vts")
        with open(p, "wb") as fh:
            fh.write(_vts_bytes(dims, xyz, f))
        paths.append(p)
    p = os.path.join(out_dir, f"{stem}_{step:06d}.vtm")
    with open(p, "wb") as fh:
        fh.write(_vtm_bytes(stem, step, len(snap)))
    paths.append(p)
    return paths


def write_solution(fs, flowname: Optional[str] = None, step: int = 0) -> List[str]:
    """Writes the case's current solution; returns the files written."""
    return _write(_snapshot(fs), flowname, step)


def write_solution_async(fs, flowname: Optional[str] = None, step: int = 0) -> cf.Future:
    """Takes the device snapshot now and writes the files on a background
    thread; the case may keep stepping meanwhile.  The future's result is the
    list of files."""
    return _writer.submit(_write, _snapshot(fs), flowname, step)


def save_restart(fs, path: str, step: int = 0) -> None:
    """Primitive variables of every block (padded, FP64) and the step number."""
    arrays = {f"prim_{b}": fs.download(b, "prim") for b in range(len(fs.case.blocks))}
    np.savez(path, step=np.int64(step), nblocks=np.int64(len(fs.case.blocks)),
             dims=np.array([b.dims for b in fs.case.blocks], dtype=np.int64), **arrays)


def load_restart(fs, path: str) -> int:
    """Uploads a restart written by save_restart into a case of the same blocks;
    returns its step number."""
    with np.load(path) as z:
        if int(z["nblocks"]) != len(fs.case.blocks) or \
                [tuple(d) for d in z["dims"]] != [tuple(b.dims) for b in fs.case.blocks]:
            raise _lib.OrionError("restart: blocks do not match the case")
        for b in range(len(fs.case.blocks)):
            fs.upload(b, "prim", z[f"prim_{b}"])
        return int(z["step"])
