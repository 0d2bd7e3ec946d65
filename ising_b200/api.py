"""Python host mirror of the reference's driver-facing routines over libisinggpu.

Names, argument meaning and error behaviour follow the Fortran routines of
SamuelJosephs/ISING (citations per function).  Where the reference calls ``error stop``
these raise :class:`IsingError`.  All compute runs in the CUDA library; nothing here
computes physics on the CPU.
"""
from __future__ import annotations

import atexit
import ctypes as C
import weakref
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import (CELL_BCC, CELL_HYPER_KAGOME, CELL_SC, DMI_BULK, DMI_INTERFACIAL, MOVE_BALL,
                   MOVE_UNIFORM, PT_EVEN_ODD, PT_RANDOM_PAIRS, ENS_ORDER_GROUPS, ENS_ORDER_PHASE, EnsembleDesc,
                   EnsSchedule, EnsemblesOptions, IsingError, MeshInfo, Params, PTOptions)

_P = C.POINTER

# Live native handles, closed in dependency order (networks and engines, PT objects, then
# meshes) when the interpreter exits: finalisers that run later, in arbitrary order and after
# the CUDA runtime has begun to shut down, must find nothing left to free.
_LIVE = {"net": weakref.WeakSet(), "eng": weakref.WeakSet(), "pt": weakref.WeakSet(), "mesh": weakref.WeakSet()}


def _close_all():
    for kind in ("net", "eng", "pt", "mesh"):
        for obj in list(_LIVE[kind]):
            try:
                obj.close()
            except Exception:
                pass


atexit.register(_close_all)


def _dp(a: np.ndarray):
    return a.ctypes.data_as(_P(C.c_double))


# ---------------------------------------------------------------- unit cells
def unit_cell(kind: int):
    """(a, b, c, ab, bc, ca, frac) of ISING_CELL_SC / _BCC (src/unit_cells.f90:7-30) /
    _HYPER_KAGOME (src/unit_cells.f90:32-77)."""
    a, b, c, ab, bc, ca = (C.c_double() for _ in range(6))
    frac = (C.c_float * 36)()
    n = C.c_int()
    _lib.call("ising_unit_cell", kind, C.byref(a), C.byref(b), C.byref(c), C.byref(ab), C.byref(bc),
              C.byref(ca), frac, C.byref(n))
    f = np.array(frac[: 3 * n.value], dtype=np.float32).reshape(n.value, 3)
    return a.value, b.value, c.value, ab.value, bc.value, ca.value, f


def bcc_unit_cell():
    return unit_cell(CELL_BCC)


def hyper_kagome_unit_cell():
    return unit_cell(CELL_HYPER_KAGOME)


def sc_unit_cell():
    return unit_cell(CELL_SC)


# ---------------------------------------------------------------- Hamiltonian
def params(J=0.0, J_prime=0.0, Dz=0.0, Dz_prime=0.0, B=0.0, K=0.0, K_axis=(0.0, 0.0, 1.0),
           zeeman_factor=1.0, include_Jp=True, dmi="interfacial", dmi_axis=None,
           legacy_neighbours=False, demag=False) -> Params:
    """Hamiltonian block.  Defaults follow calculateHeisenbergEnergy / Metropolis_mcs
    (src/energyMin.f90:86-171): Zeeman factor 1, J' on, interfacial DMI about c_hat.
    Sign convention E = +J S.S' (src/energyMin.f90:139): a ferromagnet has J < 0."""
    p = Params()
    p.J, p.J_prime, p.Dz, p.Dz_prime, p.B, p.K = J, J_prime, Dz, Dz_prime, B, K
    p.K_axis[:] = list(K_axis)
    p.zeeman_factor = zeeman_factor
    p.include_Jp = int(bool(include_Jp))
    p.dmi_mode = DMI_BULK if dmi == "bulk" else DMI_INTERFACIAL
    p.dmi_axis[:] = list(dmi_axis) if dmi_axis is not None else [0.0, 0.0, 0.0]
    p.legacy_neighbours = int(bool(legacy_neighbours))
    p.demag = int(bool(demag))
    return p


def reference_params(which: str, J, J_prime, Dz, Dz_prime, B) -> Params:
    """Conventions of one reference routine: 'local' (calculateHeisenbergEnergy,
    Metropolis_mcs) or 'total' (TotalHeisenbergEnergy: g*mu_B*B, no J', D axis z)."""
    p = Params()
    _lib.call("ising_params_reference", 0 if which == "local" else 1, J, J_prime, Dz, Dz_prime, B, C.byref(p))
    return p


# ---------------------------------------------------------------- lattice
class ChainMesh:
    """makeChainMesh (src/chainMesh.f90:729-911) on the device, with n_replicas spin buffers."""

    def __init__(self, numCellsX: int, numCellsY: int, numCellsZ: int, atoms_in_unit_cell,
                 a: float, b: float, c: float, ab_deg: float = 90.0, bc_deg: float = 90.0,
                 ca_deg: float = 90.0, distance_threshold: Optional[float] = None,
                 numShells: Optional[int] = None, n_replicas: int = 1, device: int = 0):
        frac = np.ascontiguousarray(atoms_in_unit_cell, dtype=np.float32).reshape(-1, 3)
        h = C.c_void_p()
        _lib.call("ising_mesh_create", frac.ctypes.data_as(_P(C.c_float)), frac.shape[0], numCellsX,
                  numCellsY, numCellsZ, a, b, c, ab_deg, bc_deg, ca_deg,
                  distance_threshold if distance_threshold else 0.0, numShells if numShells else 0,
                  n_replicas, device, C.byref(h))
        self._h = h
        _LIVE["mesh"].add(self)
        info = MeshInfo()
        _lib.call("ising_mesh_get_info", h, C.byref(info))
        self.info = info
        self.numAtoms = int(info.num_atoms)
        self.numCellsX, self.numCellsY, self.numCellsZ = info.nx, info.ny, info.nz
        self.n_sub = info.n_sub
        self.n_replicas = info.n_replicas
        self.checkerboard = info.checkerboard == 1
        self.layout = {0: "reference", 1: "checkerboard", 2: "octant", 3: "sublattice"}.get(info.checkerboard,
                                                                                            str(info.checkerboard))
        self.a_vec = np.array(info.a_vec[:])
        self.b_vec = np.array(info.b_vec[:])
        self.c_vec = np.array(info.c_vec[:])

    @classmethod
    def simple_cubic(cls, L: int, ny: Optional[int] = None, nz: Optional[int] = None, a: float = 1.0,
                     **kw) -> "ChainMesh":
        return cls(L, ny or L, nz or L, np.zeros((1, 3), np.float32), a, a, a, **kw)

    @property
    def handle(self):
        return self._h

    def _depend(self, obj):
        """Register a PT object or engine that must be destroyed before this mesh."""
        if not hasattr(self, "_dependents"):
            self._dependents = weakref.WeakSet()
        self._dependents.add(obj)

    def close(self):
        for d in list(getattr(self, "_dependents", ())):
            d.close()
        if getattr(self, "_h", None) and self._h.value:
            _lib.load().ising_mesh_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # spins ---------------------------------------------------------------
    def get_spins(self, replica: int = 0) -> np.ndarray:
        """atomSpins(numAtoms, 3) of one replica (FP64, widened from the device FP32)."""
        out = np.empty((3, self.numAtoms), dtype=np.float64)
        _lib.call("ising_spins_get", self._h, replica, _dp(out))
        return out.T

    def set_spins(self, spins, replica: int = 0):
        s = np.asarray(spins, dtype=np.float64).reshape(self.numAtoms, 3)
        col = np.ascontiguousarray(s.T)
        _lib.call("ising_spins_set", self._h, replica, _dp(col))

    def get_spins_async(self, host_ptr: int, replica: int = 0):
        """Queue the download of one replica's atomSpins (3 x numAtoms FP64, column-major) to
        the host address `host_ptr` (pinned memory for overlap, e.g. a pinned torch tensor's
        data_ptr()); complete after wait_spins()."""
        _lib.call("ising_spins_get_async", self._h, replica, C.cast(host_ptr, _P(C.c_double)))

    def set_spins_async(self, host_ptr: int, replica: int = 0):
        """Queue the upload of one replica from the host address `host_ptr` (same layout);
        it starts after the last queued download of that replica."""
        _lib.call("ising_spins_set_async", self._h, replica, C.cast(host_ptr, _P(C.c_double)))

    def wait_spins(self):
        """Wait for every queued transfer; raises on invalid uploaded spins."""
        _lib.call("ising_spins_wait", self._h)

    @property
    def atomSpins(self) -> np.ndarray:
        return self.get_spins(0)

    @atomSpins.setter
    def atomSpins(self, v):
        self.set_spins(v, 0)

    def set_stream(self, cuda_stream: Optional[int]):
        """Issue this mesh's device work on an external stream (e.g. a torch stream's
        .cuda_stream); None restores the mesh's own stream."""
        _lib.call("ising_mesh_set_stream", self._h, C.c_void_p(cuda_stream) if cuda_stream else None)

    def init_uniform(self, seed: int, ensemble: int = 0):
        _lib.call("ising_spins_init_uniform", self._h, seed, ensemble)

    # geometry ------------------------------------------------------------
    def positions(self) -> np.ndarray:
        out = np.empty((self.numAtoms, 3), dtype=np.float32)
        _lib.call("ising_mesh_positions", self._h, out.ctypes.data_as(_P(C.c_float)))
        return out

    def neighbours(self, atom: int, shell: int) -> np.ndarray:
        """0-based neighbour atoms: shell 0/1 = atomShells(atom+1, 1/2)%NNList, -1 = NeighborList."""
        cap = 256
        out = np.empty(cap, dtype=np.int64)
        n = C.c_int()
        _lib.call("ising_mesh_neighbours", self._h, atom, shell, out.ctypes.data_as(_P(C.c_int64)), cap, C.byref(n))
        return out[: n.value].copy()

    def colouring(self, p: Params):
        """(colour per atom, number of classes) the sweep uses for Hamiltonian p."""
        out = np.empty(self.numAtoms, dtype=np.int32)
        n = C.c_int()
        _lib.call("ising_mesh_colouring", self._h, C.byref(p), out.ctypes.data_as(_P(C.c_int)), C.byref(n))
        return out, n.value

    def derivative_list(self) -> np.ndarray:
        out = np.empty((self.numAtoms, 3, 2), dtype=np.int64)
        _lib.call("ising_mesh_derivative_list", self._h, out.ctypes.data_as(_P(C.c_int64)))
        return out


def make_chain_mesh(numCellsX, numCellsY, numCellsZ, atoms_in_unit_cell, a, b, c, ab_deg, bc_deg, ca_deg,
                    distance_threshold=None, numShells=None, n_replicas=1, device=0) -> ChainMesh:
    return ChainMesh(numCellsX, numCellsY, numCellsZ, atoms_in_unit_cell, a, b, c, ab_deg, bc_deg, ca_deg,
                     distance_threshold, numShells, n_replicas, device)


# ---------------------------------------------------------------- energies
def calculate_heisenberg_energy(mesh: ChainMesh, atomIndex: int, J, J_prime, Dz, Dz_prime, B,
                                S_proposed, demag: bool = False, replica: int = 0,
                                p: Optional[Params] = None):
    """calculateHeisenbergEnergy (src/energyMin.f90:86-171): (oldEnergy, newEnergy) of the
    1-based atomIndex for the current spin and S_proposed."""
    if p is None:
        p = reference_params("local", J, J_prime, Dz, Dz_prime, B)
        p.demag = int(bool(demag))
    sp = np.ascontiguousarray(S_proposed, dtype=np.float64)
    o, n = C.c_double(), C.c_double()
    _lib.call("ising_local_energy", mesh.handle, replica, atomIndex, C.byref(p), _dp(sp), C.byref(o), C.byref(n))
    return o.value, n.value


def local_energy_batch(mesh: ChainMesh, atoms, s_prop, p: Params, replica: int = 0):
    atoms = np.ascontiguousarray(atoms, dtype=np.int64)
    sp = np.ascontiguousarray(s_prop, dtype=np.float64).reshape(-1, 3)
    n = atoms.shape[0]
    old, new = np.empty(n), np.empty(n)
    _lib.call("ising_local_energy_batch", mesh.handle, replica, n, atoms.ctypes.data_as(_P(C.c_int64)), _dp(sp),
              C.byref(p), _dp(old), _dp(new))
    return old, new


def total_heisenberg_energy(mesh: ChainMesh, J, J_prime, Dz, Dz_prime, B, demag: bool = False,
                            replica: int = 0, p: Optional[Params] = None) -> float:
    """TotalHeisenbergEnergy (src/energyMin.f90:499-528)."""
    if p is None:
        p = reference_params("total", J, J_prime, Dz, Dz_prime, B)
        p.demag = int(bool(demag))
    e = C.c_double()
    _lib.call("ising_total_energy", mesh.handle, replica, C.byref(p), C.byref(e))
    return e.value


def observables(mesh: ChainMesh, p: Params):
    """(E[R], M[R,3]) of every replica in one device pass."""
    R = mesh.n_replicas
    e, m = np.empty(R), np.empty((R, 3))
    _lib.call("ising_observables", mesh.handle, C.byref(p), _dp(e), _dp(m))
    return e, m


# ---------------------------------------------------------------- sweeps
def metropolis_mcs(mesh: ChainMesh, beta: float, numMCSSweeps: int, J, J_prime, Dz, Dz_prime, B, r,
                   lockArray=None, demag: bool = False, replica: int = 0, seed: int = 0x15196,
                   p: Optional[Params] = None):
    """Metropolis_mcs (src/energyMin.f90:234-374) as an exact colour-class sweep on the GPU.
    r > 0 selects the ball move of radius r; lockArray is accepted and ignored."""
    if p is None:
        p = reference_params("local", J, J_prime, Dz, Dz_prime, B)
        p.demag = int(bool(demag))
    _lib.call("ising_metropolis_mcs", mesh.handle, replica, beta, numMCSSweeps, C.byref(p), r, seed)


# ---------------------------------------------------------------- winding number
def calculate_winding_number2(mesh: ChainMesh, Z_index: int, replica: int = 0) -> float:
    """calculate_winding_number2 (src/reciprocalSpaceProcesses.f90:320-364), 1-based Z_index."""
    q = C.c_double()
    _lib.call("ising_winding_number", mesh.handle, replica, Z_index, C.byref(q))
    return q.value


def demag_field(mesh: ChainMesh, replica: int = 0) -> np.ndarray:
    """calculate_demagnetisation_field (src/reciprocalSpaceProcesses.f90:202-281): the
    demagnetising field at every atom, (numAtoms, 3) FP64."""
    out = np.empty((3, mesh.numAtoms))
    _lib.call("ising_demag_field", mesh.handle, replica, _dp(out))
    return out.T


def write_demagnetisation_field_to_file(mesh: ChainMesh, filepath: str, replica: int = 0):
    """write_demagnetisation_field_to_file (src/energyMin.f90:559-583) of the field of the
    replica's current spins."""
    _lib.call("ising_write_demag_csv", mesh.handle, replica, filepath.encode())


def winding_all_slices(mesh: ChainMesh, replica: int = 0) -> np.ndarray:
    out = np.empty(mesh.numCellsZ)
    _lib.call("ising_winding_all_slices", mesh.handle, replica, _dp(out))
    return out


def calculate_winding_number_density(mesh: ChainMesh, Z_index: int, replica: int = 0) -> np.ndarray:
    """calculate_winding_number_density (rsp:438-500): (numCellsX, numCellsY) array."""
    out = np.empty(mesh.numCellsX * mesh.numCellsY)
    _lib.call("ising_winding_density", mesh.handle, replica, Z_index, _dp(out))
    return out.reshape(mesh.numCellsY, mesh.numCellsX).T


def winding_density_all_slices(mesh: ChainMesh, replica: int = 0) -> np.ndarray:
    """The densities of every z slice in one launch: (numCellsX, numCellsY, numCellsZ) array,
    slice z-1 equal to calculate_winding_number_density(mesh, z)."""
    out = np.empty(mesh.numCellsX * mesh.numCellsY * mesh.numCellsZ)
    _lib.call("ising_winding_density_all", mesh.handle, replica, _dp(out))
    return out.reshape(mesh.numCellsZ, mesh.numCellsY, mesh.numCellsX).transpose(2, 1, 0)


def set_interpolation_scale(mesh: ChainMesh, sclx: int = 10, scly: int = 10):
    """makeChainMesh's sclx, scly (src/chainMesh.f90:745-773): fine grid = (sclx*nx, scly*ny)."""
    _lib.call("ising_mesh_set_interpolation_scale", mesh.handle, int(sclx), int(scly))


def interpolation_scale(mesh: ChainMesh):
    sx, sy = C.c_int(0), C.c_int(0)
    _lib.call("ising_mesh_interpolation_scale", mesh.handle, C.byref(sx), C.byref(sy))
    return sx.value, sy.value


def calculate_winding_density_interpolated(mesh: ChainMesh, z_index: int, replica: int = 0) -> np.ndarray:
    """calculate_winding_density_interpolated (rsp:366-436): (sclx*numCellsX, scly*numCellsY)."""
    sx, sy = interpolation_scale(mesh)
    fx, fy = sx * mesh.numCellsX, sy * mesh.numCellsY
    out = np.empty(fx * fy)
    _lib.call("ising_winding_density_interpolated", mesh.handle, replica, z_index, _dp(out))
    return out.reshape(fy, fx).T


def calculate_skyrmion_number(mesh: ChainMesh, Z_index: int, q_threshold: float, particle_number: int,
                              sigma: float, replica: int = 0) -> int:
    """calculate_skyrmion_number (rsp:627-812)."""
    out = C.c_int(0)
    _lib.call("ising_skyrmion_number", mesh.handle, replica, Z_index, float(q_threshold), int(particle_number),
              float(sigma), C.byref(out))
    return out.value


def compute_skyrmion_distribution(mesh: ChainMesh, N: int, min_threshold: float, max_threshold: float,
                                  num_thresholds: int, Z_index: int, replica: int = 0) -> np.ndarray:
    """compute_skyrmion_distribution (rsp:930-983): counts of particles with charge 1..N."""
    out = np.zeros(N, dtype=np.int32)
    _lib.call("ising_skyrmion_distribution", mesh.handle, replica, int(N), float(min_threshold),
              float(max_threshold), int(num_thresholds), int(Z_index), out.ctypes.data_as(C.POINTER(C.c_int)))
    return out


def gaussian_filter_2d(array: np.ndarray, sigma: float) -> np.ndarray:
    """Gaussian_filter_2d (rsp:814-859) of a 2-D array (returns the filtered copy)."""
    a = np.asfortranarray(np.array(array, dtype=np.float64))
    _lib.call("ising_gaussian_filter_2d", a.ctypes.data_as(C.POINTER(C.c_double)), a.shape[0], a.shape[1],
              float(sigma))
    return a


def skyrmion_number_from_density(density: np.ndarray, numCellsX: int, numCellsY: int, q_threshold: float,
                                 particle_number: int, sigma: float) -> int:
    """calculate_skyrmion_number after its interpolation step, on a given fine density."""
    a = np.asfortranarray(np.asarray(density, dtype=np.float64))
    out = C.c_int(0)
    _lib.call("ising_skyrmion_number_density", a.ctypes.data_as(C.POINTER(C.c_double)), a.shape[0], a.shape[1],
              int(numCellsX), int(numCellsY), float(q_threshold), int(particle_number), float(sigma), C.byref(out))
    return out.value


def chain_mesh_statistics_full(mesh: ChainMesh, replica: int = 0):
    """chainMesh_statistics (src/PT-Utils.f90:33-66): (skyrmion_number_middle,
    winding_number_middle, winding_number_spread, magnetisation[3])."""
    sk = C.c_int(0)
    wm, ws = C.c_double(0), C.c_double(0)
    m = np.zeros(3)
    _lib.call("ising_chain_mesh_statistics", mesh.handle, replica, C.byref(sk), C.byref(wm), C.byref(ws), _dp(m))
    return sk.value, wm.value, ws.value, m


def chain_mesh_statistics(mesh: ChainMesh, replica: int = 0):
    """chainMesh_statistics (src/PT-Utils.f90:33-66) without the skyrmion count:
    (winding_number_middle, winding_number_spread, magnetisation[3])."""
    wm, ws = C.c_double(), C.c_double()
    m = np.empty(3)
    _lib.call("ising_statistics", mesh.handle, replica, C.byref(wm), C.byref(ws), _dp(m))
    return wm.value, ws.value, m


# ---------------------------------------------------------------- CSV outputs
def write_spins_to_file(mesh: ChainMesh, filename: str, append: bool = False, include_header: bool = True,
                        frame_index: Optional[int] = None, replica: int = 0):
    """write_spins_to_file (src/LLG.f90:93-172)."""
    _lib.call("ising_write_spins_csv", mesh.handle, replica, filename.encode(), int(append), int(include_header),
              -1 if frame_index is None else int(frame_index))


def write_winding_number_density(mesh: ChainMesh, filepath: str, replica: int = 0):
    """write_winding_number_density (rsp:544-580)."""
    _lib.call("ising_write_winding_density_csv", mesh.handle, replica, filepath.encode())


def pt_file_tag(J, D, B, T) -> str:
    """The (F0.4,"_",F0.4,"_",F0.4,"_",e0.4) tag of src/PT.f90:337-338."""
    buf = C.create_string_buffer(256)
    _lib.call("ising_pt_file_tag", buf, 256, J, D, B, T)
    return buf.value.decode()


def write_winding_number_density_interpolated(mesh: ChainMesh, filepath: str, replica: int = 0):
    """write_winding_number_density_interpolated (rsp:502-540)."""
    _lib.call("ising_write_winding_density_interpolated_csv", mesh.handle, replica, filepath.encode())


def frame_filename(output_dir: str, index: int) -> str:
    """trim(output_dir)//"/frame_"//I5.5//".csv" of src/ISING.f90:218."""
    buf = C.create_string_buffer(len(output_dir) + 64)
    _lib.call("ising_frame_filename", buf, len(buf), output_dir.encode(), int(index))
    return buf.value.decode()


def write_frame_info(path: str, num_frames: int, numCellsX: int, latticeParam: float):
    """info.txt of the annealing driver (src/ISING.f90:232-237)."""
    _lib.call("ising_write_frame_info", path.encode(), int(num_frames), int(numCellsX), float(latticeParam))


def write_pt_data_csv(path: str, J, D, B, T, winding_number_middle, skyrmion_number_middle,
                      winding_number_spread, magnetisation: Sequence[float]):
    """The data_<tag>.csv record of src/PT.f90:318-362."""
    m = np.ascontiguousarray(magnetisation, dtype=np.float64)
    _lib.call("ising_write_pt_data_csv", path.encode(), J, D, B, T, winding_number_middle,
              int(skyrmion_number_middle), winding_number_spread, _dp(m))


# ---------------------------------------------------------------- parallel tempering
def temperature_ladder(Tmin: float, Tmax: float, n: int) -> np.ndarray:
    """Geometric ladder T_j = Tmin (Tmax/Tmin)^((j-1)/(n-1)) (src/PT.f90:202)."""
    if n == 1:
        return np.array([Tmin])
    j = np.arange(n)
    return Tmin * (Tmax / Tmin) ** (j / (n - 1))


class ParallelTempering:
    """The PT block of src/PT.f90:193-272 on the device: replicas 0..n-1 of `mesh` start at
    temperature slots 0..n-1; exchange relabels slots (TemperatureMeshArray)."""

    def __init__(self, mesh: ChainMesh, betas, p: Params, seed: int = 0x15196, ensemble: int = 0,
                 move: int = MOVE_BALL, r: float = 0.2, scheme: int = PT_EVEN_ODD, resync_every: int = 0,
                 record: bool = False, record_capacity: int = 0, l2_group: int = 0, sweep_kernel: int = 0):
        self.mesh = mesh
        self.betas = np.ascontiguousarray(betas, dtype=np.float64)
        self.n = len(self.betas)
        self.p = p
        o = PTOptions()
        o.seed, o.ensemble, o.move, o.r, o.scheme = seed, ensemble, move, r, scheme
        o.resync_every, o.record, o.record_capacity = resync_every, int(record), record_capacity
        o.l2_group = l2_group
        o.sweep_kernel = sweep_kernel
        self.opt = o
        h = C.c_void_p()
        _lib.call("ising_pt_create", mesh.handle, self.n, _dp(self.betas), C.byref(p), C.byref(o), C.byref(h))
        self._h = h
        mesh._depend(self)
        _LIVE["pt"].add(self)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            _lib.load().ising_pt_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, sweeps_per_swap: int, rounds: int):
        _lib.call("ising_pt_run", self._h, sweeps_per_swap, rounds)

    def relax(self, n_sweeps: int):
        """Sweeps without exchange (the relax loop of src/PT.f90:276-287)."""
        _lib.call("ising_pt_relax", self._h, n_sweeps)

    def schedule(self, sweeps_per_swap: int):
        """(replicas per L2 group, colour-pass launches per round, kernel id)."""
        g, n, k = C.c_int(), C.c_int(), C.c_int()
        _lib.call("ising_pt_schedule", self._h, sweeps_per_swap, C.byref(g), C.byref(n), C.byref(k))
        return g.value, n.value, k.value

    def permutation(self) -> np.ndarray:
        out = np.empty(self.n, dtype=np.int32)
        _lib.call("ising_pt_permutation", self._h, out.ctypes.data_as(_P(C.c_int)))
        return out

    def energies(self):
        e, m = np.empty(self.n), np.empty((self.n, 3))
        _lib.call("ising_pt_energies", self._h, _dp(e), _dp(m))
        return e, m

    def resync(self):
        _lib.call("ising_pt_resync", self._h)

    def inject_stall(self, wait_ms: int = 200):
        """Test hook (octant meshes): the next run's dependency waits give up after wait_ms."""
        _lib.call("ising_pt_inject_stall", self._h, wait_ms)

    def swap_stats(self):
        att = np.zeros(max(self.n - 1, 1), dtype=np.uint64)
        acc = np.zeros(max(self.n - 1, 1), dtype=np.uint64)
        _lib.call("ising_pt_swap_stats", self._h, att.ctypes.data_as(_P(C.c_uint64)),
                  acc.ctypes.data_as(_P(C.c_uint64)))
        return att[: self.n - 1], acc[: self.n - 1]

    # learned patch move ------------------------------------------------------
    def patch_step(self, net: "ProposalNet", colour: int, offset=(0, 0, 0), slots: int = 0):
        """One class of the 2x2x2 colouring of 4^3 blocks, shifted by offset, on the
        replicas holding temperature slots 0..slots-1 (0: all)."""
        _lib.call("ising_pt_patch_step", self._h, net.handle, colour, offset[0], offset[1], offset[2], slots)

    def patch_set_scale(self, scale, drift: float = 1.0):
        """Per-slot step scale (None restores 1) and drift weight of the patch move."""
        self._drift = drift
        if scale is None:
            _lib.call("ising_pt_patch_set_scale", self._h, None, drift)
            return
        a = np.ascontiguousarray(scale, dtype=np.float32)
        assert a.size == self.n
        _lib.call("ising_pt_patch_set_scale", self._h, a.ctypes.data_as(_P(C.c_float)), drift)

    def patch_tune_scale(self, net: "ProposalNet", target: float = 0.25, iters: int = 12, init: float = 0.3,
                         seed: int = 0, drift: float = 1.0):
        """Robbins-Monro tuning of the per-slot step scale toward a target acceptance (each
        iteration is an ordinary patch step of all eight colour classes)."""
        rng = np.random.default_rng(seed)
        a = np.full(self.n, init)
        for it in range(iters):
            self.patch_set_scale(a, drift)
            p0, c0 = self.patch_stats()
            for c in range(8):
                self.patch_step(net, c, tuple(int(v) for v in rng.integers(0, 8, 3)))
            p1, c1 = self.patch_stats()
            acc = (c1 - c0) / np.maximum(p1 - p0, 1)
            a = np.clip(a * np.exp(2.0 * (acc - target) / np.sqrt(it + 1.0)), 1e-3, 2.0)
        self.patch_set_scale(a, drift)
        return a

    def patch_count(self, slots: int = 0) -> int:
        n = C.c_int64()
        _lib.call("ising_pt_patch_count", self._h, slots, C.byref(n))
        return n.value

    def patch_samples(self, colour: int, offset=(0, 0, 0), slots: int = 0, n_local: int = 20):
        """(windows [n,3,8,8,8], targets [n,64,3]) as float32 CUDA tensors."""
        import torch
        n = self.patch_count(slots)
        w = torch.empty((n, 3, 8, 8, 8), dtype=torch.float32, device="cuda")
        t = torch.empty((n, 64, 3), dtype=torch.float32, device="cuda")
        fp = lambda x: C.cast(x.data_ptr(), _P(C.c_float))
        _lib.call("ising_pt_patch_samples", self._h, colour, offset[0], offset[1], offset[2], slots, n_local, fp(w), fp(t))
        return w, t

    def patch_jump(self) -> np.ndarray:
        """Per slot: summed squared spin displacement of the accepted patch moves."""
        out = np.zeros(self.n)
        _lib.call("ising_pt_patch_jump", self._h, _dp(out))
        return out

    def patch_stats(self):
        p = np.zeros(self.n, dtype=np.uint64)
        a = np.zeros(self.n, dtype=np.uint64)
        _lib.call("ising_pt_patch_stats", self._h, p.ctypes.data_as(_P(C.c_uint64)), a.ctypes.data_as(_P(C.c_uint64)))
        return p, a

    def series(self) -> np.ndarray:
        """(n_temps, n_recorded, 4): E, |M|, Q_mid, Q_mean per recorded sweep."""
        cap = self.opt.record_capacity
        out = np.empty((self.n, cap, 4))
        n = C.c_int()
        _lib.call("ising_pt_series", self._h, _dp(out), C.byref(n))
        return out[:, : n.value, :]


_ORDER_NAMES = {0: "phase", 1: "groups", 2: "wave"}
_LOADER_NAMES = {0: "registers", 1: "staged", 2: "fused"}


class Ensembles:
    """Many PT ensembles (parameter slots of src/PT.f90:147-176) advanced together by one
    persistent kernel per launch.  `members` is a sequence of (mesh, betas, params,
    ensemble_id); each mesh must be a colour-separated simple-cubic mesh of its own."""

    def __init__(self, members, seed: int = 0x15196, move: int = MOVE_BALL, r: float = 0.2,
                 scheme: int = PT_EVEN_ODD, resync_every: int = 0, wait_timeout_ms: int = 0):
        self.members = list(members)
        self._betas = [np.ascontiguousarray(b, dtype=np.float64) for _, b, _, _ in self.members]
        descs = (EnsembleDesc * len(self.members))()
        for i, (mesh, _, p, ens) in enumerate(self.members):
            descs[i].mesh = mesh.handle
            descs[i].n_temps = len(self._betas[i])
            descs[i].betas = _dp(self._betas[i])
            descs[i].params = p
            descs[i].ensemble = ens
        o = EnsemblesOptions()
        o.seed, o.move, o.r, o.scheme, o.resync_every, o.wait_timeout_ms = seed, move, r, scheme, resync_every, wait_timeout_ms
        self.opt = o
        h = C.c_void_p()
        _lib.call("ising_ensembles_create", len(self.members), descs, C.byref(o), C.byref(h))
        self._h = h
        for mesh, *_ in self.members:
            mesh._depend(self)
        _LIVE["eng"].add(self)

    @classmethod
    def for_rank(cls, members, rank: int, world: int, sweeps: int = 1, **kw):
        """The share of `members` that one rank of a multi-GPU job runs: whole ensembles,
        balanced by sites x temperatures x sweeps (``sharding.partition_ensembles``), as an
        engine of its own with no collective between ranks (the parameter slots of
        src/PT.f90:147-176 never exchange data).  Returns (engine or None when the rank gets
        no ensemble, indices into `members`)."""
        from .sharding import members_for_rank
        idx, mine = members_for_rank(members, rank, world, sweeps)
        return (cls(mine, **kw) if mine else None), idx

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            _lib.load().ising_ensembles_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr: Optional[int]):
        _lib.call("ising_ensembles_set_stream", self._h, C.c_void_p(stream_ptr or 0))

    def run(self, sweeps_per_swap: int, rounds: int):
        _lib.call("ising_ensembles_run", self._h, sweeps_per_swap, rounds)

    def set_schedule(self, block_threads: int = 256, chunk_pairs: int = 4096, order: int = ENS_ORDER_PHASE,
                     group_bytes: int = 48_000_000, loader: int = 0):
        """loader 0: neighbours loaded per thread; 1: rows staged in shared memory by TMA
        (nz = 128 and nx % 4 == 0 in every ensemble, 256-thread blocks); 2: both colour passes
        of a sweep fused into one pass over ping-pong buffers (128..512-thread blocks of at
        least nz threads; even sweeps_per_swap)."""
        c = EnsSchedule(block_threads, chunk_pairs, order, group_bytes, 0.0, loader)
        _lib.call("ising_ensembles_set_schedule", self._h, C.byref(c))

    def schedule(self) -> dict:
        c, g, t = EnsSchedule(), C.c_int(), C.c_int64()
        _lib.call("ising_ensembles_get_schedule", self._h, C.byref(c), C.byref(g), C.byref(t))
        return {"block_threads": c.block_threads, "chunk_pairs": c.chunk_pairs,
                "order": _ORDER_NAMES.get(c.order, str(c.order)), "group_bytes": c.group_bytes,
                "loader": _LOADER_NAMES.get(c.loader, str(c.loader)),
                "ms_per_round": c.ms_per_round, "grid_blocks": g.value, "tasks_per_pass": t.value}

    def autotune(self, sweeps_per_swap: int, rounds_per_trial: int = 1):
        """Times the candidate schedules and keeps the fastest; returns the trials."""
        trials = (EnsSchedule * 64)()
        n = C.c_int()
        _lib.call("ising_ensembles_autotune", self._h, sweeps_per_swap, rounds_per_trial, trials, 64, C.byref(n))
        return [{"block_threads": t.block_threads, "chunk_pairs": t.chunk_pairs,
                 "order": _ORDER_NAMES.get(t.order, str(t.order)), "group_bytes": t.group_bytes,
                 "loader": _LOADER_NAMES.get(t.loader, str(t.loader)),
                 "ms_per_round": t.ms_per_round} for t in trials[: n.value]]

    def permutation(self, e: int) -> np.ndarray:
        out = np.empty(len(self._betas[e]), dtype=np.int32)
        _lib.call("ising_ensembles_permutation", self._h, e, out.ctypes.data_as(_P(C.c_int)))
        return out

    def energies(self, e: int):
        n = len(self._betas[e])
        en, m = np.empty(n), np.empty((n, 3))
        _lib.call("ising_ensembles_energies", self._h, e, _dp(en), _dp(m))
        return en, m

    def swap_stats(self, e: int):
        n = len(self._betas[e])
        att = np.zeros(max(n - 1, 1), dtype=np.uint64)
        acc = np.zeros(max(n - 1, 1), dtype=np.uint64)
        _lib.call("ising_ensembles_swap_stats", self._h, e, att.ctypes.data_as(_P(C.c_uint64)),
                  acc.ctypes.data_as(_P(C.c_uint64)))
        return att[: n - 1], acc[: n - 1]

    def resync(self):
        _lib.call("ising_ensembles_resync", self._h)

    def set_resync(self, every: int):
        """FP64 recomputation of the accumulators after each `every` rounds of run(),
        counted from this call (0: never)."""
        _lib.call("ising_ensembles_set_resync", self._h, every)

    def inject_stall(self, e: int):
        """Test hook: the next run's rounds >= 1 of ensemble e wait for a flag nothing sets."""
        _lib.call("ising_ensembles_inject_stall", self._h, e)


class ProposalNet:
    """The learned patch proposal's network on one GPU (tensor-core forward, backward and
    Adam).  Windows are float32 CUDA tensors [n, 3, 8, 8, 8]; outputs [n, 64, 4]."""

    def __init__(self, device: int = 0, max_batch: int = 1024, seed: int = 1):
        h = C.c_void_p()
        _lib.call("ising_net_create", device, max_batch, seed, C.byref(h))
        self._h = h
        _LIVE["net"].add(self)
        self.max_batch = max_batch
        self.n_params = _lib.load().ising_net_param_count()

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            _lib.load().ising_net_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_params(self) -> np.ndarray:
        out = np.empty(self.n_params, dtype=np.float32)
        _lib.call("ising_net_get_params", self._h, out.ctypes.data_as(_P(C.c_float)))
        return out

    def set_params(self, flat):
        a = np.ascontiguousarray(flat, dtype=np.float32)
        assert a.size == self.n_params
        _lib.call("ising_net_set_params", self._h, a.ctypes.data_as(_P(C.c_float)))

    @staticmethod
    def _fp(t):
        return C.cast(t.data_ptr(), _P(C.c_float))

    def forward(self, windows):
        import torch
        w = windows.contiguous()
        out = torch.empty((w.shape[0], 64, 4), dtype=torch.float32, device=w.device)
        _lib.call("ising_net_forward", self._h, self._fp(w), w.shape[0], self._fp(out))
        return out

    def loss_grad(self, windows, targets):
        w, t = windows.contiguous(), targets.contiguous()
        loss = C.c_double()
        g = np.empty(self.n_params, dtype=np.float32)
        _lib.call("ising_net_loss_grad", self._h, self._fp(w), self._fp(t), w.shape[0], C.byref(loss),
                  g.ctypes.data_as(_P(C.c_float)))
        return loss.value, g

    def train_step(self, windows, targets, lr: float = 1e-3) -> float:
        w, t = windows.contiguous(), targets.contiguous()
        loss = C.c_double()
        _lib.call("ising_net_train_step", self._h, self._fp(w), self._fp(t), w.shape[0], lr, C.byref(loss))
        return loss.value
