"""Python host side of the B200 flow solver: a ctypes binding of the C ABI in
``include/minicombust_flow.h`` and a ``FlowSolver`` class that mirrors the
reference's ``minicombust::flow::FlowSolver<double>`` interface
(include/flow/FlowSolver.hpp:95-147, 1003-1048): construct from a mesh and a
time step, call ``timestep()``, read fields.

Every compute call goes to the sm_100a library ``lib/libmcflow.so``; there is
no CPU fallback.  Loading the library on a machine without a GPU works (mesh
building and parameter defaults are host code), but creating a solver then
fails with ``FlowError`` (MC_ERR_CUDA).
"""
import ctypes
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "lib", "libmcflow.so")

c_u64 = ctypes.c_uint64
c_dbl = ctypes.c_double
c_int = ctypes.c_int
c_long = ctypes.c_long
c_vp = ctypes.c_void_p

MC_OK = 0
MC_ERR_ARG = -1
MC_ERR_CUDA = -2
MC_ERR_NOT_CONVERGED = -3
MC_ERR_NONFINITE = -4
MC_ERR_MESH = -5
MC_ERR_NOMEM = -6
MC_ERR_UNSUPPORTED = -7
MC_ERR_TIMEOUT = -8

MODE_COMPAT, MODE_SIMPLE = 0, 1
PSOLVER_PCG_JACOBI, PSOLVER_PCG_AMG = 0, 1
PRECISION_FP64, PRECISION_FP32_REFINED = 0, 1
REORDER_NONE, REORDER_RCM = 0, 1
GUESS_ZERO, GUESS_PREVIOUS, GUESS_LEARNED = 0, 1, 2
SNAPSHOT_MAGIC = b"MCSNAP01"
HEADER_PATH = os.path.join(os.path.dirname(_PKG), "include", "minicombust_flow.h")


def header_define(name, path=HEADER_PATH):
    """Integer value of a ``#define`` in the C header (ctypes cannot see macros)."""
    with open(path) as f:
        for line in f:
            parts = line.split()
            if len(parts) >= 3 and parts[0] == "#define" and parts[1] == name:
                return int(parts[2])
    raise KeyError(f"{name} is not defined in {path}")


def read_snapshots(path):
    """Records of a snapshot file as a read-only array [records][4][cells]
    (rhs projected to mean zero, diagonal, previous correction, correction)."""
    with open(path, "rb") as f:
        head = f.read(64)
    if head[:8] != SNAPSHOT_MAGIC:
        raise ValueError(f"{path}: not a snapshot file")
    version, cells, fields, dtype = np.frombuffer(head[8:24], dtype=np.uint32)
    records = int(np.frombuffer(head[24:32], dtype=np.uint64)[0])
    if version != 1 or fields != 4 or dtype != 0:
        raise ValueError(f"{path}: unsupported snapshot layout")
    return np.memmap(path, dtype=np.float32, mode="r", offset=64, shape=(records, 4, int(cells)))
SYSTEM_MOMENTUM, SYSTEM_PRESSURE, SYSTEM_TEMPERATURE, SYSTEM_MOMENTUM_V, SYSTEM_MOMENTUM_W = 0, 1, 2, 3, 4

FIELDS = {"U": 0, "V": 1, "W": 2, "P": 3, "PP": 4, "TE": 5, "ED": 6, "TP": 7, "TEM": 8,
          "FUL": 9, "PRO": 10, "VARF": 11, "VARP": 12}


class MeshView(ctypes.Structure):
    """mc_mesh_view: the reference Mesh<T> arrays (Mesh.hpp:86-106)."""
    _fields_ = [("cells", c_u64), ("faces", c_u64), ("points", c_u64),
                ("points_xyz", ctypes.POINTER(c_dbl)), ("cell_nodes", ctypes.POINTER(c_u64)),
                ("face_cells", ctypes.POINTER(c_u64)), ("cell_faces", ctypes.POINTER(c_u64)),
                ("cell_neighbours", ctypes.POINTER(c_u64)), ("cell_centers", ctypes.POINTER(c_dbl)),
                ("boundary_types", c_u64 * 6)]


class FlowParams(ctypes.Structure):
    _fields_ = [("mode", c_int), ("delta", c_dbl), ("density", c_dbl), ("viscosity", c_dbl),
                ("inlet_u", c_dbl), ("pressure0", c_dbl), ("temperature0", c_dbl),
                ("urf_momentum", c_dbl), ("urf_pressure", c_dbl), ("urf_temperature", c_dbl),
                ("flux_corr", c_dbl), ("u_rtol", c_dbl), ("p_rtol", c_dbl), ("max_iters", c_int),
                ("pressure_solver", c_int), ("precision", c_int), ("initial_guess", c_int), ("device", c_int),
                ("amg_sweeps", c_int), ("amg_omega", c_dbl), ("amg_alpha", c_dbl), ("ir_inner_rtol", c_dbl),
                ("reorder", c_int), ("ir_inner_rtol_bicg", c_dbl),
                ("amg_cheb_ratio", c_dbl), ("transport_scalars", c_int), ("ir_line_steps", c_int)]


class IterStats(ctypes.Structure):
    _fields_ = [("momentum_iters", c_int * 3), ("temperature_iters", c_int), ("pressure_solves", c_int),
                ("pressure_iters_total", c_int), ("pressure_iters_first", c_int),
                ("pressure_correction_max_first", c_dbl), ("pressure_rel_residual", c_dbl),
                ("mass_imbalance", c_dbl), ("guess_choice_first", c_int), ("guess_rel_residual_first", c_dbl),
                ("pressure_rel_residual_first", c_dbl), ("scalar_iters", c_int * 6)]

    def as_dict(self):
        return {"momentum_iters": list(self.momentum_iters), "temperature_iters": self.temperature_iters,
                "pressure_solves": self.pressure_solves, "pressure_iters_total": self.pressure_iters_total,
                "pressure_iters_first": self.pressure_iters_first,
                "pressure_correction_max_first": self.pressure_correction_max_first,
                "pressure_rel_residual": self.pressure_rel_residual, "mass_imbalance": self.mass_imbalance,
                "guess_choice_first": self.guess_choice_first,
                "guess_rel_residual_first": self.guess_rel_residual_first,
                "pressure_rel_residual_first": self.pressure_rel_residual_first,
                "scalar_iters": list(self.scalar_iters)}


class FlowError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(message)
        self.status = status


# Exported entry points and their signatures (restype, argtypes).
_SIGNATURES = {
    "mc_flow_default_params": (None, [ctypes.POINTER(FlowParams), c_int]),
    "mc_flow_create": (c_int, [ctypes.POINTER(MeshView), ctypes.POINTER(FlowParams), ctypes.POINTER(c_vp)]),
    "mc_flow_destroy": (c_int, [c_vp]),
    "mc_flow_set_field": (c_int, [c_vp, c_int, c_vp]),
    "mc_flow_get_field": (c_int, [c_vp, c_int, c_vp]),
    "mc_flow_get_gradient": (c_int, [c_vp, c_int, c_vp]),
    "mc_flow_set_sources": (c_int, [c_vp, c_vp]),
    "mc_flow_get_face_array": (c_int, [c_vp, c_int, c_vp]),
    "mc_flow_get_cell_order": (c_int, [c_vp, c_vp]),
    "mc_flow_write_vtk": (c_int, [c_vp, ctypes.c_char_p, c_int]),
    "mc_flow_ingest_particles": (c_int, [c_vp, ctypes.c_int64, c_vp, c_vp]),
    "mc_flow_get_sources": (c_int, [c_vp, c_vp]),
    "mc_flow_set_sources_device": (c_int, [c_vp, c_vp]),
    "mc_flow_interpolate_nodes": (c_int, [c_vp, ctypes.c_int64, c_vp, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64),
                                          c_vp, c_vp]),
    "mc_flow_checkpoint_write": (c_int, [c_vp, ctypes.c_char_p]),
    "mc_flow_checkpoint_read": (c_int, [c_vp, ctypes.c_char_p]),
    "mc_flow_set_guess_params": (c_int, [c_vp, c_vp, c_int]),
    "mc_flow_snapshot_open": (c_int, [c_vp, ctypes.c_char_p, c_int]),
    "mc_flow_snapshot_close": (c_int, [c_vp]),
    "mc_flow_get_cell_array": (c_int, [c_vp, c_int, c_vp]),
    "mc_flow_get_csr": (c_int, [c_vp, c_int, ctypes.POINTER(c_int), ctypes.POINTER(c_int), c_vp, c_vp, c_vp, c_vp]),
    "mc_flow_simple_iteration": (c_int, [c_vp, ctypes.POINTER(IterStats)]),
    "mc_flow_timestep": (c_int, [c_vp, ctypes.POINTER(IterStats)]),
    "mc_flow_stage_gradients": (c_int, [c_vp]),
    "mc_flow_stage_set_up_field": (c_int, [c_vp]),
    "mc_flow_stage_momentum": (c_int, [c_vp, ctypes.POINTER(IterStats)]),
    "mc_flow_stage_pressure": (c_int, [c_vp, ctypes.POINTER(IterStats)]),
    "mc_flow_stage_temperature": (c_int, [c_vp, ctypes.POINTER(IterStats)]),
    "mc_flow_stage_scalar": (c_int, [c_vp, c_int, ctypes.POINTER(IterStats)]),
    "mc_flow_set_timing": (c_int, [c_vp, c_int]),
    "mc_flow_kernel_count": (c_int, []),
    "mc_flow_kernel_name": (ctypes.c_char_p, [c_int]),
    "mc_flow_get_kernel_times": (c_int, [c_vp, c_vp, c_vp]),
    "mc_flow_reset_kernel_times": (c_int, [c_vp]),
    "mc_flow_stream": (c_vp, [c_vp]),
    "mc_flow_launch_count": (c_long, [c_vp]),
    "mc_flow_last_error": (ctypes.c_char_p, [c_vp]),
    "mc_status_string": (ctypes.c_char_p, [c_int]),
    "mc_solve_bicgstab_noalloc": (c_int, [c_int, c_vp, c_vp, c_vp, c_vp, c_vp, c_dbl, c_int, c_vp,
                                          ctypes.POINTER(c_int)]),
    "mc_mesh_box_create": (c_int, [c_u64, c_u64, c_u64, c_dbl, c_dbl, c_dbl, ctypes.POINTER(MeshView)]),
    "mc_mesh_box_destroy": (None, [ctypes.POINTER(MeshView)]),
    "mc_mesh_rcm_order": (c_int, [ctypes.POINTER(MeshView), c_vp]),
}

_lib = None


def library():
    """Load lib/libmcflow.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} is missing: run `python -m minicombust_app_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def default_params(mode=MODE_SIMPLE, **overrides):
    p = FlowParams()
    library().mc_flow_default_params(ctypes.byref(p), mode)
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise AttributeError(k)
        setattr(p, k, v)
    return p


def _check(status, handle=None, what=""):
    if status != MC_OK:
        L = library()
        msg = L.mc_status_string(status).decode()
        if handle:
            detail = L.mc_flow_last_error(handle).decode()
            if detail:
                msg += ": " + detail
        raise FlowError(status, f"{what}: {msg}" if what else msg)


class Mesh:
    """Mesh arrays in the reference layout, owned by numpy."""

    def __init__(self, points, cell_nodes, face_cells, cell_faces, cell_neighbours, cell_centers, boundary_types,
                 dims=None):
        self.points = np.ascontiguousarray(points, dtype=np.float64)
        self.cell_nodes = np.ascontiguousarray(cell_nodes, dtype=np.uint64)
        self.face_cells = np.ascontiguousarray(face_cells, dtype=np.uint64)
        self.cell_faces = np.ascontiguousarray(cell_faces, dtype=np.uint64)
        self.cell_neighbours = np.ascontiguousarray(cell_neighbours, dtype=np.uint64)
        self.cell_centers = np.ascontiguousarray(cell_centers, dtype=np.float64)
        self.boundary_types = np.ascontiguousarray(boundary_types, dtype=np.uint64)
        self.dims = dims

    @property
    def n_cells(self):
        return self.cell_nodes.shape[0]

    @property
    def n_faces(self):
        return self.face_cells.shape[0]

    @classmethod
    def box(cls, ex, ey, ez, lx, ly, lz):
        """The reference's load_mesh box (mesh_examples.cpp:120-571), built by the library."""
        L = library()
        mv = MeshView()
        _check(L.mc_mesh_box_create(ex, ey, ez, lx, ly, lz, ctypes.byref(mv)), what="mc_mesh_box_create")
        try:
            N, F, P = mv.cells, mv.faces, mv.points
            out = cls(np.ctypeslib.as_array(mv.points_xyz, shape=(P * 3,)).reshape(P, 3).copy(),
                      np.ctypeslib.as_array(mv.cell_nodes, shape=(N * 8,)).reshape(N, 8).copy(),
                      np.ctypeslib.as_array(mv.face_cells, shape=(F * 2,)).reshape(F, 2).copy(),
                      np.ctypeslib.as_array(mv.cell_faces, shape=(N * 6,)).reshape(N, 6).copy(),
                      np.ctypeslib.as_array(mv.cell_neighbours, shape=(N * 6,)).reshape(N, 6).copy(),
                      np.ctypeslib.as_array(mv.cell_centers, shape=(N * 3,)).reshape(N, 3).copy(),
                      np.array(list(mv.boundary_types), dtype=np.uint64), dims=(ex, ey, ez))
        finally:
            L.mc_mesh_box_destroy(ctypes.byref(mv))
        return out

    def rcm_order(self):
        """Reverse Cuthill-McKee cell order (new-to-old) used by REORDER_RCM."""
        out = np.empty(self.n_cells, dtype=np.int32)
        mv = self.view()
        _check(library().mc_mesh_rcm_order(ctypes.byref(mv), _ptr(out)), what="mc_mesh_rcm_order")
        return out

    def renumbered(self, cell_new_to_old):
        """The same mesh with its cells renumbered (faces keep their order;
        an internal face whose cells change order swaps its roles, as the
        reference requires cell0 < cell1)."""
        n2o = np.asarray(cell_new_to_old, dtype=np.int64)
        N = self.n_cells
        o2n = np.empty(N, dtype=np.int64)
        o2n[n2o] = np.arange(N)
        nb = self.cell_neighbours[n2o].copy()
        internal = nb < N
        nb[internal] = o2n[nb[internal].astype(np.int64)].astype(np.uint64)
        fc = self.face_cells.astype(np.int64)
        c0 = o2n[fc[:, 0]]
        c1 = np.where(fc[:, 1] < N, o2n[np.minimum(fc[:, 1], N - 1)], fc[:, 1])
        swap = (fc[:, 1] < N) & (c1 < c0)
        fc_new = np.stack([np.where(swap, c1, c0), np.where(swap, c0, c1)], axis=1)
        return Mesh(self.points, self.cell_nodes[n2o], fc_new.astype(np.uint64), self.cell_faces[n2o], nb,
                    self.cell_centers[n2o], self.boundary_types)

    def view(self):
        mv = MeshView()
        mv.cells, mv.faces, mv.points = self.n_cells, self.n_faces, self.points.shape[0]
        mv.points_xyz = self.points.ctypes.data_as(ctypes.POINTER(c_dbl))
        mv.cell_nodes = self.cell_nodes.ctypes.data_as(ctypes.POINTER(c_u64))
        mv.face_cells = self.face_cells.ctypes.data_as(ctypes.POINTER(c_u64))
        mv.cell_faces = self.cell_faces.ctypes.data_as(ctypes.POINTER(c_u64))
        mv.cell_neighbours = self.cell_neighbours.ctypes.data_as(ctypes.POINTER(c_u64))
        mv.cell_centers = self.cell_centers.ctypes.data_as(ctypes.POINTER(c_dbl))
        for i in range(6):
            mv.boundary_types[i] = int(self.boundary_types[i])
        return mv


def _ptr(a):
    return a.ctypes.data_as(c_vp)


class FlowSolver:
    """Mirror of minicombust::flow::FlowSolver<double> over the C ABI.

    ``FlowSolver(mesh, delta)`` builds the solver (FlowSolver.hpp:147);
    ``timestep()`` runs three SIMPLE passes (FlowSolver.inl:3148-3356);
    ``simple_iteration()`` runs one.  Fields are read and written in the
    reference layout: ``cells + 6`` doubles with the boundary-side slots last.
    """

    def __init__(self, mesh, delta=None, params=None, mode=MODE_SIMPLE):
        self.L = library()
        self.mesh = mesh
        p = params if params is not None else default_params(mode)
        if delta is not None:
            p.delta = delta
        self.params = p
        self.N = mesh.n_cells
        self.F = mesh.n_faces
        self._mv = mesh.view()
        h = c_vp()
        _check(self.L.mc_flow_create(ctypes.byref(self._mv), ctypes.byref(p), ctypes.byref(h)), what="mc_flow_create")
        self.h = h
        self.compute_time = 0.0
        self.last_stats = IterStats()

    def close(self):
        if getattr(self, "h", None):
            self.L.mc_flow_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # --- fields ---------------------------------------------------------
    def field(self, name):
        a = np.empty(self.N + 6)
        _check(self.L.mc_flow_get_field(self.h, FIELDS[name], _ptr(a)), self.h, "get_field")
        return a

    def set_field(self, name, values):
        a = np.ascontiguousarray(values, dtype=np.float64)
        if a.shape != (self.N + 6,):
            raise ValueError(f"field must have {self.N + 6} values")
        _check(self.L.mc_flow_set_field(self.h, FIELDS[name], _ptr(a)), self.h, "set_field")

    def gradient(self, name):
        a = np.empty((self.N, 3))
        _check(self.L.mc_flow_get_gradient(self.h, FIELDS[name], _ptr(a)), self.h, "get_gradient")
        return a

    def set_sources(self, particle_terms):
        a = np.ascontiguousarray(particle_terms, dtype=np.float64)
        if a.shape != (self.N, 5):
            raise ValueError("particle terms must be [cells][5]")
        _check(self.L.mc_flow_set_sources(self.h, _ptr(a)), self.h, "set_sources")

    def ingest_particles(self, cells, terms):
        """Particle rows (cell id, particle_aos) in arrival order become the
        source terms (the flow side of update_flow_field)."""
        c = np.ascontiguousarray(cells, dtype=np.uint64)
        t = np.ascontiguousarray(terms, dtype=np.float64)
        if t.shape != (c.shape[0], 5):
            raise ValueError("terms must be [rows][5]")
        _check(self.L.mc_flow_ingest_particles(self.h, c.shape[0], _ptr(c), _ptr(t)), self.h, "ingest_particles")

    def set_sources_device(self, ptr):
        """Sources from device memory [5][cells] (a device pointer, e.g.
        tensor.data_ptr()), ordered on the handle's stream."""
        _check(self.L.mc_flow_set_sources_device(self.h, ptr), self.h, "set_sources_device")

    def sources(self):
        a = np.empty((self.N, 5))
        _check(self.L.mc_flow_get_sources(self.h, _ptr(a)), self.h, "get_sources")
        return a

    def interpolate_nodes(self, cells):
        """(node ids ascending, [nodes][5] = vel.x, vel.y, vel.z, pressure, temp)
        for the nodes of the given cells."""
        c = np.ascontiguousarray(cells, dtype=np.uint64)
        n = ctypes.c_int64()
        _check(self.L.mc_flow_interpolate_nodes(self.h, c.shape[0], _ptr(c), 0, ctypes.byref(n), None, None),
               self.h, "interpolate_nodes")
        ids = np.empty(n.value, dtype=np.uint64)
        vals = np.empty((n.value, 5))
        _check(self.L.mc_flow_interpolate_nodes(self.h, c.shape[0], _ptr(c), n.value, ctypes.byref(n), _ptr(ids),
                                                _ptr(vals)), self.h, "interpolate_nodes")
        return ids, vals

    def face_array(self, which):
        width = {4: 2, 5: 3, 6: 3}.get(which, 1)
        a = np.empty((self.F, width))
        _check(self.L.mc_flow_get_face_array(self.h, which, _ptr(a)), self.h, "get_face_array")
        return a if width > 1 else a[:, 0]

    def set_guess_params(self, params):
        """Parameters of the learned guess (MC_GUESS_LEARNED), as from gnn.GuessNet.params()."""
        p = np.ascontiguousarray(params, dtype=np.float32)
        _check(self.L.mc_flow_set_guess_params(self.h, _ptr(p), len(p)), self.h, "set_guess_params")

    def snapshot_open(self, path, max_records):
        _check(self.L.mc_flow_snapshot_open(self.h, os.fsencode(path), int(max_records)), self.h, "snapshot_open")

    def snapshot_close(self):
        _check(self.L.mc_flow_snapshot_close(self.h), self.h, "snapshot_close")

    def output_data(self, timestep, prefix="out/flow/minicombust"):
        """FlowSolver::output_data (FlowSolver.inl:18-23): the VTK flow file of
        this timestep, as the reference's VisitWriter writes it."""
        _check(self.L.mc_flow_write_vtk(self.h, os.fsencode(prefix), int(timestep)), self.h, "write_vtk")
        return f"{prefix}_flow0_timestep{int(timestep)}.vtk"

    def checkpoint(self, path):
        _check(self.L.mc_flow_checkpoint_write(self.h, os.fsencode(path)), self.h, "checkpoint_write")

    def resume(self, path):
        _check(self.L.mc_flow_checkpoint_read(self.h, os.fsencode(path)), self.h, "checkpoint_read")

    def cell_order(self):
        """The handle's internal cell order: new-to-old ids (identity unless reordered)."""
        a = np.empty(self.N, dtype=np.int32)
        _check(self.L.mc_flow_get_cell_order(self.h, _ptr(a)), self.h, "get_cell_order")
        return a

    def cell_array(self, which):
        a = np.empty(self.N)
        _check(self.L.mc_flow_get_cell_array(self.h, which, _ptr(a)), self.h, "get_cell_array")
        return a

    def csr(self, system):
        n, nnz = c_int(), c_int()
        _check(self.L.mc_flow_get_csr(self.h, system, ctypes.byref(n), ctypes.byref(nnz), None, None, None, None),
               self.h, "get_csr")
        rp = np.empty(n.value + 1, dtype=np.int32)
        col = np.empty(nnz.value, dtype=np.int32)
        val = np.empty(nnz.value)
        rhs = np.empty(n.value)
        _check(self.L.mc_flow_get_csr(self.h, system, ctypes.byref(n), ctypes.byref(nnz), _ptr(rp), _ptr(col),
                                      _ptr(val), _ptr(rhs)), self.h, "get_csr")
        return rp, col, val, rhs

    # --- stepping ---------------------------------------------------------
    def simple_iteration(self, check=True):
        rc = self.L.mc_flow_simple_iteration(self.h, ctypes.byref(self.last_stats))
        if check:
            _check(rc, self.h, "simple_iteration")
        return rc

    def timestep(self, check=True):
        rc = self.L.mc_flow_timestep(self.h, ctypes.byref(self.last_stats))
        if check:
            _check(rc, self.h, "timestep")
        return rc

    def stage(self, name):
        s = self.last_stats
        fn = {"gradients": lambda: self.L.mc_flow_stage_gradients(self.h),
              "set_up_field": lambda: self.L.mc_flow_stage_set_up_field(self.h),
              "momentum": lambda: self.L.mc_flow_stage_momentum(self.h, ctypes.byref(s)),
              "pressure": lambda: self.L.mc_flow_stage_pressure(self.h, ctypes.byref(s)),
              "temperature": lambda: self.L.mc_flow_stage_temperature(self.h, ctypes.byref(s))}[name]
        _check(fn(), self.h, name)

    def stage_scalar(self, name):
        """Scalar_solve for one transported field: TE, ED, TEM, FUL, PRO, VARF or VARP."""
        _check(self.L.mc_flow_stage_scalar(self.h, FIELDS[name], ctypes.byref(self.last_stats)), self.h,
               f"stage_scalar({name})")

    # --- instrumentation --------------------------------------------------
    def set_timing(self, on):
        _check(self.L.mc_flow_set_timing(self.h, 1 if on else 0), self.h, "set_timing")

    def kernel_times(self):
        n = self.L.mc_flow_kernel_count()
        ms = np.zeros(n)
        cnt = np.zeros(n, dtype=np.int64)
        _check(self.L.mc_flow_get_kernel_times(self.h, _ptr(ms), _ptr(cnt)), self.h, "get_kernel_times")
        return {self.L.mc_flow_kernel_name(i).decode(): (float(ms[i]), int(cnt[i])) for i in range(n)}

    def reset_kernel_times(self):
        _check(self.L.mc_flow_reset_kernel_times(self.h), self.h, "reset_kernel_times")

    def launch_count(self):
        return int(self.L.mc_flow_launch_count(self.h))

    def stream(self):
        return self.L.mc_flow_stream(self.h)
