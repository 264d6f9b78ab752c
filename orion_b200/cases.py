"""Case builder: bump-channel grids, block splits, BC topology and flow parameters.

A case is everything the per-step solver path needs as input: per-block grid
point coordinates, the BC region list of every block in ORION's own form
(``BCRegion`` in src/bc/BCData.hpp:8-54, read from ``.inp`` files by
src/bc/BCReader.cpp:31-182), and the flow parameters that the hot path reads
(``core::Params``, src/core/Params.hpp:9-120).

Geometry (all configurations): x in [0,2] uniform, z in [0,0.5] uniform, the
lower wall carries a Gaussian bump h(x) = H exp(-((x-1)/0.1)^2) and y is
stretched from the bump to y=1 with a tanh law clustered at the wall,
    y(i,j) = h(x_i) + (1 - h(x_i)) * (1 + tanh(beta*(eta_j - 1)) / tanh(beta)),
eta_j = j/(NJ-1), beta = 2.

BCs, in file order per block: j-min adiabatic no-slip wall (type 2), i-min and
i-max characteristic far field (4), j-max far field (4), k-min and k-max
symmetry (3).  Faces inside the domain become point-matched 1-to-1 interfaces
(type -1) with identity orientation.  The per-block region order is
[j-min, i-min, i-max, j-max, k-min, k-max]; physical BCs are applied in that
order (src/bc/PhysicalBC.cpp:587), which matters on shared edges.

``Case.write_reference_inputs`` writes param.dat / grid.x / bc.inp / noise.txt
in the reference's own file formats so the reference reads the same case.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

NG = 3  # ghost layers; fixed by the scheme (src/preprocess/FlowField.cpp:9-16)
MIN_BLOCK_DIM = 12  # smallest block extent the line closures support

BC_INTERFACE = -1
BC_WALL = 2
BC_SYMMETRY = 3
BC_FARFIELD = 4
BC_FREESTREAM = 5
BC_EXTRAPOLATION = 6

# face order of the region list of every block
FACES = ("jmin", "imin", "imax", "jmax", "kmin", "kmax")
PHYSICAL_TYPE = {"jmin": BC_WALL, "imin": BC_FARFIELD, "imax": BC_FARFIELD,
                 "jmax": BC_FARFIELD, "kmin": BC_SYMMETRY, "kmax": BC_SYMMETRY}
OPPOSITE = {"imin": "imax", "imax": "imin", "jmin": "jmax", "jmax": "jmin",
            "kmin": "kmax", "kmax": "kmin"}


@dataclass
class Region:
    """One BC window of a block, 1-based inclusive point ranges (BCRegion)."""
    s_st: Tuple[int, int, int]
    s_ed: Tuple[int, int, int]
    bctype: int
    t_st: Tuple[int, int, int] = (0, 0, 0)
    t_ed: Tuple[int, int, int] = (0, 0, 0)
    nbt: int = -1      # target block, 1-based (interfaces only)
    ibcwin: int = 0    # target region, 1-based (interfaces only)

    def normal_dir(self) -> int:
        """1=i, 2=j, 3=k (BCReader.cpp:126-146)."""
        for d in range(3):
            if self.s_st[d] == self.s_ed[d]:
                return d + 1
        return 0

    def side(self, dims: Sequence[int]) -> int:
        """-1 min face, +1 max face, 0 internal cut (BCReader.cpp:126-146)."""
        d = self.normal_dir() - 1
        if d < 0:
            return 0
        if self.s_st[d] == 1:
            return -1
        if self.s_st[d] == dims[d]:
            return 1
        return 0


@dataclass
class Block:
    idim: int
    jdim: int
    kdim: int
    x: np.ndarray  # shape (kdim, jdim, idim): i fastest in memory
    y: np.ndarray
    z: np.ndarray
    regions: List[Region] = field(default_factory=list)

    @property
    def dims(self) -> Tuple[int, int, int]:
        return (self.idim, self.jdim, self.kdim)

    @property
    def padded(self) -> Tuple[int, int, int]:
        return (self.idim + 2 * NG, self.jdim + 2 * NG, self.kdim + 2 * NG)

    @property
    def npoints(self) -> int:
        return self.idim * self.jdim * self.kdim


@dataclass
class FlowParams:
    """The inputs of the hot path (names follow core::Params)."""
    moo: float = 0.5
    reynolds: float = 1000.0
    cfl: float = 2.0
    twall: float = 0.0
    tref: float = 288.15
    pref: float = 101325.0
    attack: float = 0.0
    sideslip: float = 0.0
    nvis: int = 1
    method: int = 1
    ntmst: int = 0
    gcl: int = 1
    csrv: int = 1
    gamma: float = 1.4   # setup_perfect_gas_air (src/preprocess/Inflow.cpp:15-48)
    prl: float = 0.72

    # --- derived exactly as init_inflow does (src/preprocess/Inflow.cpp:300-459) ---
    @property
    def attack_rad(self) -> float:
        return self.attack * 3.14159265358979323846 / 180.0

    @property
    def sideslip_rad(self) -> float:
        return self.sideslip * 3.14159265358979323846 / 180.0

    @property
    def uoo(self) -> float:
        return math.cos(self.attack_rad) * math.cos(self.sideslip_rad)

    @property
    def voo(self) -> float:
        return math.sin(self.attack_rad) * math.cos(self.sideslip_rad)

    @property
    def woo(self) -> float:
        return math.sin(self.sideslip_rad)

    roo: float = 1.0
    too: float = 1.0

    @property
    def poo(self) -> float:
        return 1.0 / (self.gamma * self.moo * self.moo)

    @property
    def visc(self) -> float:
        return 110.4 / self.tref


@dataclass
class Case:
    name: str
    blocks: List[Block]
    params: FlowParams
    noise_seed: int = 0
    noise_amp: float = 0.01
    nsteps: int = 1

    @property
    def npoints(self) -> int:
        return sum(b.npoints for b in self.blocks)

    @property
    def padded_points(self) -> int:
        return sum(int(np.prod(b.padded)) for b in self.blocks)

    # ------------------------------------------------------------------
    def write_reference_inputs(self, path: str) -> None:
        """param.dat / grid.x / bc.inp / noise.txt in ORION's formats."""
        os.makedirs(path, exist_ok=True)
        write_param_dat(os.path.join(path, "param.dat"), self.params, self.nsteps)
        write_plot3d(os.path.join(path, "grid.x"), self.blocks)
        write_bc_inp(os.path.join(path, "bc.inp"), self.blocks)
        with open(os.path.join(path, "noise.txt"), "w") as f:
            f.write(f"{self.noise_seed} {self.noise_amp!r}\n")


# ---------------------------------------------------------------------------
# geometry
# ---------------------------------------------------------------------------

def bump_grid(NI: int, NJ: int, NK: int, height: float, beta: float = 2.0):
    """Global bump-channel grid; arrays shaped (NK, NJ, NI)."""
    i = np.arange(NI, dtype=np.float64)
    j = np.arange(NJ, dtype=np.float64)
    k = np.arange(NK, dtype=np.float64)
    x1 = 2.0 * i / (NI - 1)
    z1 = 0.5 * k / (NK - 1)
    eta = j / (NJ - 1)
    h = height * np.exp(-((x1 - 1.0) / 0.1) ** 2)
    frac = 1.0 + np.tanh(beta * (eta - 1.0)) / math.tanh(beta)
    y2 = h[None, :] + (1.0 - h[None, :]) * frac[:, None]        # (NJ, NI)
    x = np.broadcast_to(x1[None, None, :], (NK, NJ, NI)).copy()
    y = np.broadcast_to(y2[None, :, :], (NK, NJ, NI)).copy()
    z = np.broadcast_to(z1[:, None, None], (NK, NJ, NI)).copy()
    return x, y, z


def even_splits(n: int, parts: int) -> List[int]:
    """Shared-plane split points 0 = s0 < s1 < ... < s_parts = n-1."""
    return [round(p * (n - 1) / parts) for p in range(parts + 1)]


def uneven_splits(n: int, parts: int, rng: np.random.Generator, ratio: float = 3.0) -> List[int]:
    """Seeded split points whose block extents differ by up to ``ratio``."""
    if parts == 1:
        return [0, n - 1]
    cells = n - 1
    for _ in range(1000):
        w = rng.uniform(1.0, ratio, size=parts)
        w = w / w.sum() * cells
        ext = np.maximum(np.round(w).astype(int), MIN_BLOCK_DIM - 1)
        ext[-1] = cells - ext[:-1].sum()
        if ext.min() >= MIN_BLOCK_DIM - 1 and ext.max() <= ratio * ext.min() + 1:
            return [0] + [int(v) for v in np.cumsum(ext)]
    return even_splits(n, parts)


def split_case(name: str, x: np.ndarray, y: np.ndarray, z: np.ndarray,
               si: Sequence[int], sj: Sequence[int], sk: Sequence[int],
               params: FlowParams, nsteps: int, noise_seed: int, noise_amp: float = 0.01,
               physical: Optional[Dict[str, int]] = None) -> Case:
    """Cut a global grid into blocks at the given shared planes and build the
    region lists (physical BCs on the domain boundary, interfaces inside).
    `physical` overrides the BC type of domain faces (PHYSICAL_TYPE)."""
    types = {**PHYSICAL_TYPE, **(physical or {})}
    nbi, nbj, nbk = len(si) - 1, len(sj) - 1, len(sk) - 1
    blocks: List[Block] = []

    def bid(a, b, c):
        return a + nbi * (b + nbj * c)

    for c in range(nbk):
        for b in range(nbj):
            for a in range(nbi):
                i0, i1 = si[a], si[a + 1]
                j0, j1 = sj[b], sj[b + 1]
                k0, k1 = sk[c], sk[c + 1]
                sl = (slice(k0, k1 + 1), slice(j0, j1 + 1), slice(i0, i1 + 1))
                blk = Block(i1 - i0 + 1, j1 - j0 + 1, k1 - k0 + 1,
                            np.ascontiguousarray(x[sl]), np.ascontiguousarray(y[sl]),
                            np.ascontiguousarray(z[sl]))
                if min(blk.dims) < MIN_BLOCK_DIM:
                    raise ValueError(f"block extent {blk.dims} below {MIN_BLOCK_DIM}")
                blocks.append(blk)

    for c in range(nbk):
        for b in range(nbj):
            for a in range(nbi):
                blk = blocks[bid(a, b, c)]
                for f in FACES:
                    s_st, s_ed = face_window(blk.dims, f)
                    nb = neighbour(a, b, c, f, nbi, nbj, nbk)
                    if nb is None:
                        blk.regions.append(Region(s_st, s_ed, types[f]))
                    else:
                        tgt = blocks[bid(*nb)]
                        t_st, t_ed = face_window(tgt.dims, OPPOSITE[f])
                        blk.regions.append(Region(s_st, s_ed, BC_INTERFACE, t_st, t_ed,
                                                  nbt=bid(*nb) + 1,
                                                  ibcwin=FACES.index(OPPOSITE[f]) + 1))
    return Case(name, blocks, params, noise_seed=noise_seed, noise_amp=noise_amp, nsteps=nsteps)


def face_window(dims, face):
    ni, nj, nk = dims
    lo = [1, 1, 1]
    hi = [ni, nj, nk]
    d = "ijk".index(face[0])
    if face.endswith("min"):
        hi[d] = 1
    else:
        lo[d] = dims[d]
    return tuple(lo), tuple(hi)


def neighbour(a, b, c, face, nbi, nbj, nbk):
    d = "ijk".index(face[0])
    step = -1 if face.endswith("min") else 1
    idx = [a, b, c]
    idx[d] += step
    lim = (nbi, nbj, nbk)[d]
    if idx[d] < 0 or idx[d] >= lim:
        return None
    return tuple(idx)


# ---------------------------------------------------------------------------
# named configurations
# ---------------------------------------------------------------------------

def bump_case(name: str, NI: int, NJ: int, NK: int, *, height: float = 0.05,
              split: Tuple[int, int, int] = (1, 1, 1), uneven_seed: Optional[int] = None,
              moo: float = 0.5, reynolds: float = 1000.0, nsteps: int = 1,
              noise_seed: int = 0, noise_amp: float = 0.01, cfl: float = 2.0,
              physical: Optional[Dict[str, int]] = None, nvis: int = 1, twall: float = 0.0,
              attack: float = 0.0, method: int = 1) -> Case:
    """A bump channel split into blocks.  physical: BC type per domain face
    (default PHYSICAL_TYPE); nvis 0 = Euler; twall > 0 = isothermal walls;
    attack in degrees; method 0 skips the wall-normal averaging."""
    x, y, z = bump_grid(NI, NJ, NK, height)
    if uneven_seed is None:
        si, sj, sk = (even_splits(n, p) for n, p in zip((NI, NJ, NK), split))
    else:
        rng = np.random.default_rng(uneven_seed)
        si, sj, sk = (uneven_splits(n, p, rng) for n, p in zip((NI, NJ, NK), split))
    params = FlowParams(moo=moo, reynolds=reynolds, cfl=cfl, nvis=nvis, twall=twall, attack=attack, method=method)
    return split_case(name, x, y, z, si, sj, sk, params, nsteps, noise_seed, noise_amp, physical=physical)


def config(n: int, nsteps: Optional[int] = None) -> Case:
    """The benchmark configurations: 0 single block 97x49x33 M0.5 Re1e3;
    1 eight blocks 193x97x65; 2 27 uneven blocks 289x161x65 M0.7 Re1e4;
    3 64 uneven blocks 385x257x129 M0.8 Re1e5 bump 0.08."""
    if n == 0:
        c = bump_case("c0_97x49x33", 97, 49, 33, nsteps=200, noise_seed=0)
    elif n == 1:
        c = bump_case("c1_193x97x65_8blk", 193, 97, 65, split=(2, 2, 2), nsteps=300, noise_seed=1)
    elif n == 2:
        c = bump_case("c2_289x161x65_27blk", 289, 161, 65, split=(3, 3, 3), uneven_seed=2,
                      moo=0.7, reynolds=1.0e4, nsteps=500, noise_seed=2)
    elif n == 3:
        c = bump_case("c3_385x257x129_64blk", 385, 257, 129, height=0.08, split=(4, 4, 4),
                      uneven_seed=3, moo=0.8, reynolds=1.0e5, nsteps=1000, noise_seed=3)
    else:
        raise ValueError(n)
    if nsteps is not None:
        c.nsteps = nsteps
    return c


def small_case(name: str = "small", dims=(25, 17, 13), split=(1, 1, 1), nsteps: int = 3,
               moo: float = 0.5, reynolds: float = 1000.0, noise_seed: int = 7,
               uneven_seed: Optional[int] = None, height: float = 0.05, **flow) -> Case:
    """A case small enough for the CPU oracle to step in well under a second.
    `flow`: the optional bump_case settings (physical, nvis, twall, attack, method)."""
    return bump_case(name, *dims, height=height, split=split, uneven_seed=uneven_seed, moo=moo,
                     reynolds=reynolds, nsteps=nsteps, noise_seed=noise_seed, **flow)


# ---------------------------------------------------------------------------
# reference file formats
# ---------------------------------------------------------------------------

def _f(v: float) -> str:
    return repr(float(v))


def write_param_dat(path: str, p: FlowParams, nsteps: int) -> None:
    """Fortran-namelist parameters (src/core/Params.cpp:103-275)."""
    txt = f"""$inflow
  moo = {_f(p.moo)}
  attack = {_f(p.attack)}
  sideslip = {_f(p.sideslip)}
  reynolds = {_f(p.reynolds)}
  twall = {_f(p.twall)}
  height = -1.0
  tref = {_f(p.tref)}
  pref = {_f(p.pref)}
  rref = 0.0
  ndim = 3
/
$force
  nwholefield = 1
  lfref = 1.0
  lref = 1.0
/
$control
  nstart = 0
  nomax = {nsteps}
  method = {p.method}
/
$step
  ntmst = {p.ntmst}
  cfl = {_f(p.cfl)}
/
$flowtype
  nvis = {p.nvis}
  nchem = 0
  ntmodel = 1
/
$technic
  nlhs = 21
  nscheme = 41
  nflux = 3
  efix = 0
  csrv = {p.csrv}
/
$gcl_cic
  gcl = {p.gcl}
/
"""
    with open(path, "w") as f:
        f.write(txt)


def _record(f, payload: bytes) -> None:
    n = np.array([len(payload)], dtype="<u4").tobytes()
    f.write(n)
    f.write(payload)
    f.write(n)


def write_plot3d(path: str, blocks: Sequence[Block]) -> None:
    """Multi-block Plot3D, Fortran sequential records (Plot3DReader.cpp:88-156)."""
    with open(path, "wb") as f:
        _record(f, np.array([len(blocks)], dtype="<i4").tobytes())
        for b in blocks:
            _record(f, np.array([b.idim, b.jdim, b.kdim], dtype="<i4").tobytes())
        for b in blocks:
            _record(f, np.concatenate([b.x.ravel(), b.y.ravel(), b.z.ravel()]).astype("<f8").tobytes())


def write_bc_inp(path: str, blocks: Sequence[Block]) -> None:
    """ORION BC file, marker 1976, one rank owns every block (BCReader.cpp:31-182)."""
    lines = ["1976", "1", str(len(blocks))]
    for n, b in enumerate(blocks):
        lines.append("1")
        lines.append(f"{b.idim} {b.jdim} {b.kdim}")
        lines.append(f"blk{n + 1}")
        lines.append(str(len(b.regions)))
        for r in b.regions:
            lines.append(" ".join(str(v) for v in (r.s_st[0], r.s_ed[0], r.s_st[1], r.s_ed[1],
                                                   r.s_st[2], r.s_ed[2], r.bctype)))
            if r.bctype < 0:
                lines.append(" ".join(str(v) for v in (r.t_st[0], r.t_ed[0], r.t_st[1], r.t_ed[1],
                                                       r.t_st[2], r.t_ed[2], r.nbt, r.ibcwin)))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


# ---------------------------------------------------------------------------
# readers of the same formats (case ingestion from the reference's own files)
# ---------------------------------------------------------------------------

def read_param_dat(path: str):
    """(FlowParams, nomax) from a Fortran-namelist param.dat (Params.cpp:103-275):
    `$group` ... `/` blocks of `key = value`; quotes, commas and Fortran `d`
    exponents are accepted.  Only user-given freestream conditions
    (height < 0) are supported, as the configurations use."""
    kv = {}
    with open(path) as f:
        for raw in f:
            line = raw.split("!", 1)[0].strip()
            if not line or line.startswith("$") or line.startswith("&") or line == "/":
                continue
            for part in line.rstrip(",").split(","):
                if "=" not in part:
                    continue
                k, v = part.split("=", 1)
                kv[k.strip().lower()] = v.strip().strip("'\"")

    def num(key, default, cast=float):
        if key not in kv:
            return default
        return cast(float(kv[key].lower().replace("d", "e")))

    if num("height", -1.0) >= 0.0:
        raise ValueError("param.dat: height >= 0 (standard-atmosphere conditions) is not supported")
    p = FlowParams(moo=num("moo", 0.5), reynolds=num("reynolds", 1000.0), cfl=num("cfl", 2.0),
                   twall=num("twall", 0.0), tref=num("tref", 288.15), pref=num("pref", 101325.0),
                   attack=num("attack", 0.0), sideslip=num("sideslip", 0.0), nvis=num("nvis", 1, int),
                   method=num("method", 1, int), ntmst=num("ntmst", 0, int), gcl=num("gcl", 1, int),
                   csrv=num("csrv", 1, int))
    return p, num("nomax", 1, int)


def _read_records(f):
    while True:
        head = f.read(4)
        if not head:
            return
        n = int(np.frombuffer(head, "<u4")[0])
        payload = f.read(n)
        if len(payload) != n or f.read(4) != head:
            raise ValueError("Plot3D: truncated or mismatched Fortran record")
        yield payload


def read_plot3d(path: str) -> List[Block]:
    """Blocks (coordinates only) from a multi-block Plot3D file in Fortran
    sequential records, the layout Plot3DReader.cpp:88-156 reads."""
    with open(path, "rb") as f:
        recs = _read_records(f)
        nb = int(np.frombuffer(next(recs), "<i4")[0])
        dims = [tuple(int(v) for v in np.frombuffer(next(recs), "<i4")) for _ in range(nb)]
        blocks = []
        for (ni, nj, nk) in dims:
            xyz = np.frombuffer(next(recs), "<f8").reshape(3, nk, nj, ni)
            blocks.append(Block(ni, nj, nk, xyz[0].copy(), xyz[1].copy(), xyz[2].copy(), []))
    return blocks


def read_bc_inp(path: str, blocks: Sequence[Block]) -> None:
    """Region lists from an ORION BC file (marker 1976, BCReader.cpp:31-182),
    appended to the blocks in file order.  Index ranges keep their signs (the
    interface orientation of analyze_bc_connect, BCPreprocess.cpp:16-192)."""
    with open(path) as f:
        lines = [ln.strip() for ln in f if ln.strip()]
    pos = 0

    def ints(n):
        nonlocal pos
        v = [int(t) for t in lines[pos].split()]
        pos += 1
        if len(v) != n:
            raise ValueError(f"bc file line {pos}: expected {n} integers")
        return v

    if int(lines[0]) != 1976:
        raise ValueError("bc file: marker 1976 expected")
    pos = 2  # marker, processes in the file
    nb = ints(1)[0]
    if nb != len(blocks):
        raise ValueError(f"bc file: {nb} blocks, grid has {len(blocks)}")
    for b in blocks:
        ints(1)  # owning process
        dims = ints(3)
        if tuple(dims) != b.dims:
            raise ValueError(f"bc file: block dims {dims} differ from the grid's {b.dims}")
        pos += 1  # block name
        for _ in range(ints(1)[0]):
            v = ints(7)
            r = Region((v[0], v[2], v[4]), (v[1], v[3], v[5]), v[6])
            if v[6] < 0:
                t = ints(8)
                r = Region(r.s_st, r.s_ed, v[6], (t[0], t[2], t[4]), (t[1], t[3], t[5]), t[6], t[7])
            b.regions.append(r)


def read_case(path: str, name: Optional[str] = None) -> Case:
    """A case from a directory in the reference's formats: param.dat, grid.x,
    bc.inp, and the optional noise.txt (seed, amplitude) of this package."""
    params, nsteps = read_param_dat(os.path.join(path, "param.dat"))
    blocks = read_plot3d(os.path.join(path, "grid.x"))
    read_bc_inp(os.path.join(path, "bc.inp"), blocks)
    seed, amp = 0, 0.0
    npath = os.path.join(path, "noise.txt")
    if os.path.exists(npath):
        with open(npath) as f:
            t = f.read().split()
            seed, amp = int(t[0]), float(t[1])
    return Case(name or os.path.basename(os.path.normpath(path)), blocks, params, noise_seed=seed,
                noise_amp=amp, nsteps=nsteps)


# ---------------------------------------------------------------------------
# seeded noise (same sequence as the oracle driver)
# ---------------------------------------------------------------------------

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)


def splitmix64_uniform(seed: int, start: int, count: int) -> np.ndarray:
    """Draws start+1 .. start+count of splitmix64(seed) as doubles in [0,1)."""
    with np.errstate(over="ignore"):
        n = np.arange(start + 1, start + count + 1, dtype=np.uint64)
        z = np.uint64(seed) + n * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
