"""Frame sources: seeded synthetic FCC frames and file-backed trajectories.

A frame is the raw input of one configuration, before the layout step:
``xyz`` (N, 3) float32 positions as a trajectory stores them (not folded),
``types`` (N,) int32 LAMMPS-style type ids (1-based), ``box`` (3,) float32
orthorhombic edge lengths, and optionally ``charges`` (N,) float32 per-atom
charges (the NetCDF variable ``q``, read as default real by netcdf.f90:404-408).  This is what ``read_nc_cfg`` hands to
``select_ncdfinput`` in the reference (src/core/netcdf.f90:173-550).

The synthetic generator places 4 atoms per cubic FCC cell of edge
``a = (4/density)**(1/3)``, displaces each atom by i.i.d. Gaussian noise of
standard deviation ``sigma * a`` per axis, optionally re-places a fraction of
atoms uniformly in the box, and assigns types by a seeded shuffle with given
ratios.  Species identity is fixed per trajectory (seed), displacements differ
per frame (seed, frame).  With ``charges`` given per type, atoms carry that
charge plus an optional seeded per-atom offset (``charge_jitter``, fixed per
trajectory), so both species-constant and per-atom charge sets can be made.
"""
from __future__ import annotations

import dataclasses
import os
from typing import Iterator, Optional, Sequence

import numpy as np


@dataclasses.dataclass
class Frame:
    xyz: np.ndarray      # (N, 3) float32
    types: np.ndarray    # (N,) int32, 1-based type ids
    box: np.ndarray      # (3,) float32
    charges: Optional[np.ndarray] = None  # (N,) float32
    time: Optional[float] = None          # the trajectory's time (NetCDF variable "time") of this frame

    @property
    def n(self) -> int:
        return int(self.xyz.shape[0])


@dataclasses.dataclass
class FCCSpec:
    """Seeded synthetic trajectory of FCC-derived frames."""
    cells: tuple = (10, 10, 10)          # FCC cells per axis
    density: float = 0.8                 # number density
    sigma: float = 0.12                  # Gaussian displacement, units of the cubic cell edge a
    fractions: tuple = (1.0,)            # species ratios (normalised), types 1..nsp
    replace_frac: float = 0.0            # fraction of atoms re-placed uniformly at random
    remove: int = 0                      # atoms removed by a seeded draw (to hit a target N)
    seed: int = 1234
    charges: Optional[tuple] = None      # charge per type 1..nsp (None: no charges)
    charge_jitter: float = 0.0           # std. dev. of a seeded per-atom charge offset

    @property
    def a(self) -> float:
        return (4.0 / self.density) ** (1.0 / 3.0)

    @property
    def box(self) -> np.ndarray:
        return (np.asarray(self.cells, dtype=np.float64) * self.a).astype(np.float32)

    @property
    def n(self) -> int:
        c = self.cells
        return 4 * c[0] * c[1] * c[2] - self.remove

    def _lattice(self) -> np.ndarray:
        c = self.cells
        basis = np.array([[0.0, 0.0, 0.0], [0.5, 0.5, 0.0],
                          [0.5, 0.0, 0.5], [0.0, 0.5, 0.5]])
        ix, iy, iz = np.meshgrid(np.arange(c[0]), np.arange(c[1]), np.arange(c[2]),
                                 indexing="ij")
        origins = np.stack([ix.ravel(), iy.ravel(), iz.ravel()], axis=1).astype(np.float64)
        pos = (origins[:, None, :] + basis[None, :, :]).reshape(-1, 3) * self.a
        return pos

    def _identity(self):
        """Kept-atom index and type per atom; identical for every frame."""
        rng = np.random.default_rng([self.seed, 0x5eed])
        ntot = 4 * self.cells[0] * self.cells[1] * self.cells[2]
        keep = np.arange(ntot)
        if self.remove:
            drop = rng.choice(ntot, size=self.remove, replace=False)
            keep = np.setdiff1d(keep, drop)
        n = keep.size
        fr = np.asarray(self.fractions, dtype=np.float64)
        fr = fr / fr.sum()
        counts = np.floor(fr * n + 0.5).astype(np.int64)
        counts[-1] = n - counts[:-1].sum()
        types = np.repeat(np.arange(1, len(fr) + 1, dtype=np.int32), counts)
        rng.shuffle(types)
        return keep, types

    def _base(self):
        """Kept lattice sites and types, computed once per spec (every frame shares them)."""
        key = (self.cells, self.density, self.fractions, self.remove, self.seed)
        cache = self.__dict__.get("_base_cache")
        if cache is None or cache[0] != key:
            keep, types = self._identity()
            cache = (key, self._lattice()[keep], types)
            self.__dict__["_base_cache"] = cache
        return cache[1], cache[2]

    def frame(self, index: int) -> Frame:
        base, types = self._base()
        pos = base.copy()
        rng = np.random.default_rng([self.seed, 1 + index])
        pos = pos + rng.normal(0.0, self.sigma * self.a, size=pos.shape)
        box = self.box.astype(np.float64)
        if self.replace_frac > 0:
            m = int(round(self.replace_frac * pos.shape[0]))
            idx = rng.choice(pos.shape[0], size=m, replace=False)
            pos[idx] = rng.uniform(0.0, 1.0, size=(m, 3)) * box
        return Frame(xyz=pos.astype(np.float32), types=types.copy(),
                     box=self.box.copy(), charges=self._charges(types))

    def _charges(self, types: np.ndarray) -> Optional[np.ndarray]:
        if self.charges is None:
            return None
        q = np.asarray(self.charges, np.float64)[types - 1]
        if self.charge_jitter > 0:
            rng = np.random.default_rng([self.seed, 0xc4a7])
            q = q + rng.normal(0.0, self.charge_jitter, size=q.shape)
        return q.astype(np.float32)

    def frames(self, count: int, start: int = 0) -> Iterator[Frame]:
        for i in range(start, start + count):
            yield self.frame(i)


def random_walk_frames(spec: FCCSpec, count: int, step_sigma: float, seed: int = 11,
                       time_step: float = 1.0) -> Iterator[Frame]:
    """A seeded trajectory in which every atom of ``spec.frame(0)`` takes Gaussian steps of standard
    deviation ``step_sigma`` per axis between frames (positions are not folded: atoms leave the box
    and the layout folds them back); ``time`` = frame index * time_step."""
    fr0 = spec.frame(0)
    pos = fr0.xyz.astype(np.float64)
    rng = np.random.default_rng([seed, 0xd1f])
    for f in range(count):
        if f:
            pos = pos + rng.normal(0.0, step_sigma, size=pos.shape)
        yield Frame(xyz=pos.astype(np.float32), types=fr0.types.copy(), box=fr0.box.copy(),
                    charges=None if fr0.charges is None else fr0.charges.copy(), time=float(f * time_step))


# Named workloads (shapes of the benchmark configurations).
def c1_spec(seed: int = 1) -> FCCSpec:
    """N=4000 single species, cubic L=17.0998, sigma=0.12 a."""
    return FCCSpec(cells=(10, 10, 10), density=0.8, sigma=0.12, fractions=(1.0,), seed=seed)


def c2_spec(seed: int = 2) -> FCCSpec:
    """N=62,500 binary 80:20, L=42.75, sigma=0.1 a."""
    return FCCSpec(cells=(25, 25, 25), density=0.8, sigma=0.1, fractions=(0.8, 0.2), seed=seed)


def c3_spec(seed: int = 3) -> FCCSpec:
    """N=1,000,188 three species 50:30:20, L=107.73, sigma=0.1 a, 2% re-placed."""
    return FCCSpec(cells=(63, 63, 63), density=0.8, sigma=0.1, fractions=(0.5, 0.3, 0.2),
                   replace_frac=0.02, seed=seed)


def c4_spec(seed: int = 4) -> FCCSpec:
    """N=4,000,000 slab 1:1:4 (63x63x252 cells, 752 removed), 50:50."""
    return FCCSpec(cells=(63, 63, 252), density=0.8, sigma=0.1, fractions=(0.5, 0.5),
                   remove=752, seed=seed)


WORKLOADS = {"c1": c1_spec, "c2": c2_spec, "c3": c3_spec, "c4": c4_spec}


def _frame_charges(var, f: int) -> Optional[np.ndarray]:
    if var is None:
        return None
    v = np.asarray(var[f] if len(var.shape) == 2 else var[:], np.float32)
    return np.ascontiguousarray(v)


class NpzTrajectory:
    """Frames stored as ``coordinates`` (F, N, 3), ``cell_lengths`` (F, 3), ``type`` (F, N) or (N,),
    and optionally ``q`` (F, N) or (N,) charges and ``time`` (F,)."""

    time_units = "lj"
    time_scale = 1.0

    def __init__(self, path: str):
        self._z = np.load(path)

    def __len__(self) -> int:
        return int(self._z["coordinates"].shape[0])

    def frame(self, f: int) -> Frame:
        """Frame f (0-based)."""
        z = self._z
        types = z["type"] if "type" in z else None
        t = np.ones(z["coordinates"].shape[1], np.int32) if types is None else (
            types[f] if types.ndim == 2 else types)
        return Frame(xyz=np.asarray(z["coordinates"][f], np.float32), types=np.asarray(t, np.int32),
                     box=np.asarray(z["cell_lengths"][f], np.float32),
                     charges=_frame_charges(z["q"] if "q" in z else None, f),
                     time=float(z["time"][f]) if "time" in z else None)

    def __iter__(self) -> Iterator[Frame]:
        for f in range(len(self)):
            yield self.frame(f)


class NetCDFTrajectory:
    """AMBER-convention trajectory (``coordinates``, ``cell_lengths``, optional ``type``, ``q`` and
    ``time`` with its ``units`` and ``scale_factor`` attributes, read as netcdf.f90:432-448 does).

    Uses netCDF4 when importable (every netCDF format), else scipy's reader for the classic
    formats CDF-1 and CDF-2 (64-bit offset).  A NETCDF4 (HDF5-based) file, as the reference's
    tools/lammpstrj_to_netcdf.py writes, needs netCDF4; without it the file is refused with the
    conversion command (netCDF-C's ``nccopy -k 64-bit-offset``) in the message.
    """

    HDF5_SIGNATURE = b"\x89HDF\r\n\x1a\n"

    def __init__(self, path: str):
        self._ds = None
        try:  # pragma: no cover - netCDF4 is not installed in this image
            from netCDF4 import Dataset  # type: ignore
            self._ds = Dataset(path)
            self._v = self._ds.variables
        except ImportError:
            with open(path, "rb") as f:
                head = f.read(8)
            if head == self.HDF5_SIGNATURE:
                raise ValueError(
                    f"{path}: a NETCDF4 (HDF5) file, which needs the netCDF4 package (not installed). Convert it "
                    f"to the 64-bit-offset classic format with 'nccopy -k 64-bit-offset {path} out.nc', or write "
                    f"it with format=\"NETCDF3_64BIT_OFFSET\" in the converter")
            from scipy.io import netcdf_file
            self._ds = netcdf_file(path, "r", mmap=False)
            self._v = self._ds.variables
        self.time_units, self.time_scale = "lj", 1.0
        if "time" in self._v:
            tv = self._v["time"]
            u = getattr(tv, "units", b"lj")
            self.time_units = (u.decode() if isinstance(u, bytes) else str(u)).strip()
            self.time_scale = float(getattr(tv, "scale_factor", 1.0))

    def __len__(self) -> int:
        return int(self._v["coordinates"].shape[0])

    def frame(self, f: int) -> Frame:
        """Frame f (0-based)."""
        v = self._v
        xyz = np.asarray(v["coordinates"][f], dtype=np.float32)
        t = np.asarray(v["type"][f], np.int32) if "type" in v else np.ones(xyz.shape[0], np.int32)
        return Frame(xyz=xyz, types=t, box=np.asarray(v["cell_lengths"][f], np.float32),
                     charges=_frame_charges(v["q"] if "q" in v else None, f),
                     time=float(v["time"][f]) if "time" in v else None)

    def __iter__(self) -> Iterator[Frame]:
        for f in range(len(self)):
            yield self.frame(f)


def tstep_of(traj) -> float:
    """Time per unit of the trajectory's time variable, in ps for real/metal units (common.cuf:399-412):
    scale_factor * 0.001 for femtoseconds, scale_factor for picoseconds, scale_factor otherwise."""
    if traj.time_units == "femtosecond":
        return traj.time_scale * 0.001
    return traj.time_scale


def open_trajectory(path: str):
    ext = os.path.splitext(path)[1].lower()
    if ext == ".npz":
        return NpzTrajectory(path)
    return NetCDFTrajectory(path)


def write_npz_trajectory(path: str, frames: Sequence[Frame]) -> None:
    extra = {}
    if frames[0].charges is not None:
        extra["q"] = np.stack([f.charges for f in frames])
    np.savez(path, coordinates=np.stack([f.xyz for f in frames]),
             cell_lengths=np.stack([f.box for f in frames]),
             type=np.stack([f.types for f in frames]), **extra)


def write_netcdf_trajectory(path: str, frames: Sequence[Frame]) -> None:
    """Classic NetCDF (CDF-2) file with the AMBER-convention variables the reference reads:
    coordinates (frame, atom, spatial), cell_lengths (frame, cell_spatial), type (frame, atom), and
    q (frame, atom) when the frames carry charges."""
    from scipy.io import netcdf_file
    nf = len(frames)
    n = frames[0].n
    with netcdf_file(path, "w", version=2) as nc:
        nc.Conventions = b"AMBER"
        nc.ConventionVersion = b"1.0"
        nc.createDimension("frame", nf)
        nc.createDimension("atom", n)
        nc.createDimension("spatial", 3)
        nc.createDimension("cell_spatial", 3)
        c = nc.createVariable("coordinates", "f4", ("frame", "atom", "spatial"))
        L = nc.createVariable("cell_lengths", "f4", ("frame", "cell_spatial"))
        t = nc.createVariable("type", "i4", ("frame", "atom"))
        q = nc.createVariable("q", "f4", ("frame", "atom")) if frames[0].charges is not None else None
        tv = nc.createVariable("time", "f4", ("frame",)) if frames[0].time is not None else None
        if tv is not None:
            tv.units = b"picosecond"
        for k, f in enumerate(frames):
            c[k] = f.xyz
            L[k] = f.box
            t[k] = f.types
            if q is not None:
                q[k] = f.charges
            if tv is not None:
                tv[k] = f.time
