"""ctypes bindings to the two CPU checkers built under oracle/.

Test infrastructure only (the product never imports this module):
  * ``Oracle``    -- the project's C restatement of the SIMPLE pass
                     (oracle/liboracle.so, sources oracle/mc_oracle.{c,h}).
  * ``Reference`` -- the reference's own CPU FlowSolver compiled from its
                     sources against single-rank MPI/PETSc shims
                     (oracle/_ref/libmcref.so, harness oracle/ref_harness.cpp).
"""
import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libmcref.so")

c_u64 = ctypes.c_uint64
c_dbl = ctypes.c_double
c_int = ctypes.c_int
c_vp = ctypes.c_void_p

FIELDS = {"U": 0, "V": 1, "W": 2, "P": 3, "PP": 4, "TE": 5, "ED": 6, "TP": 7, "TEM": 8,
          "FUL": 9, "PRO": 10, "VARF": 11, "VARP": 12}
COMPAT, SIMPLE = 0, 1


def _ptr(a):
    return a.ctypes.data_as(c_vp)


class MeshArrays:
    """Mesh arrays in the reference layout (Mesh.hpp:86-106)."""

    def __init__(self, ex, ey, ez, points, cells, faces, cell_faces, cell_neighbours, cell_centers, boundary_types):
        self.ex, self.ey, self.ez = ex, ey, ez
        self.points = points
        self.cells = cells
        self.faces = faces
        self.cell_faces = cell_faces
        self.cell_neighbours = cell_neighbours
        self.cell_centers = cell_centers
        self.boundary_types = boundary_types

    @property
    def n_cells(self):
        return self.cells.shape[0]

    @property
    def n_faces(self):
        return self.faces.shape[0]


class _McoParams(ctypes.Structure):
    _fields_ = [("mode", c_int), ("delta", c_dbl), ("density", c_dbl), ("viscosity", c_dbl),
                ("inlet_u", c_dbl), ("pressure0", c_dbl), ("temperature0", c_dbl),
                ("urf_momentum", c_dbl), ("urf_pressure", c_dbl), ("urf_temperature", c_dbl),
                ("flux_corr", c_dbl), ("u_rtol", c_dbl), ("p_rtol", c_dbl), ("max_iters", c_int),
                ("scalars", c_int)]


class _McoMesh(ctypes.Structure):
    _fields_ = [("ex", c_u64), ("ey", c_u64), ("ez", c_u64), ("cells", c_u64), ("faces", c_u64),
                ("points", c_u64), ("points_xyz", ctypes.POINTER(c_dbl)),
                ("cell_nodes", ctypes.POINTER(c_u64)), ("face_cells", ctypes.POINTER(c_u64)),
                ("cell_faces", ctypes.POINTER(c_u64)), ("cell_neighbours", ctypes.POINTER(c_u64)),
                ("cell_centers", ctypes.POINTER(c_dbl)), ("boundary_types", c_u64 * 6)]


class _McoStats(ctypes.Structure):
    _fields_ = [("momentum_iters", c_int * 3), ("temperature_iters", c_int), ("pressure_solves", c_int),
                ("pressure_iters_total", c_int), ("pressure_iters_first", c_int),
                ("pressure_correction_max_first", c_dbl), ("mass_imbalance", c_dbl), ("scalar_iters", c_int * 6)]


_oracle_lib = None


def oracle_lib():
    global _oracle_lib
    if _oracle_lib is None:
        L = ctypes.CDLL(ORACLE_SO)
        L.mco_default_params.argtypes = [ctypes.POINTER(_McoParams), c_int]
        L.mco_mesh_box.argtypes = [c_u64, c_u64, c_u64, c_dbl, c_dbl, c_dbl, ctypes.POINTER(_McoMesh)]
        L.mco_mesh_free.argtypes = [ctypes.POINTER(_McoMesh)]
        L.mco_create.argtypes = [ctypes.POINTER(_McoMesh), ctypes.POINTER(_McoParams)]
        L.mco_create.restype = c_vp
        L.mco_destroy.argtypes = [c_vp]
        for fn in ("mco_set_field", "mco_get_field", "mco_get_grad", "mco_get_cell_array", "mco_get_face_array",
                   "mco_get_rhs"):
            getattr(L, fn).argtypes = [c_vp, c_int, c_vp]
        L.mco_set_sources.argtypes = [c_vp, c_vp]
        L.mco_get_csr.argtypes = [c_vp, c_int, ctypes.POINTER(c_int), ctypes.POINTER(c_int), c_vp, c_vp, c_vp]
        for fn in ("mco_pass", "mco_stage_calculate_uvw", "mco_stage_calculate_pressure",
                   "mco_stage_scalar_temperature"):
            getattr(L, fn).argtypes = [c_vp]
            getattr(L, fn).restype = c_int
        for fn in ("mco_stage_gradients", "mco_stage_set_up_field"):
            getattr(L, fn).argtypes = [c_vp]
        L.mco_set_threads.argtypes = [c_int]
        L.mco_stage_scalar.argtypes = [c_vp, c_int]
        L.mco_stage_scalar.restype = c_int
        L.mco_get_stats.argtypes = [c_vp, ctypes.POINTER(_McoStats)]
        L.mco_inlet_effective_viscosity.argtypes = [c_vp]
        L.mco_inlet_effective_viscosity.restype = c_dbl
        L.mco_phi_length.argtypes = [c_vp]
        L.mco_phi_length.restype = c_u64
        _oracle_lib = L
    return _oracle_lib


def oracle_params(mode=COMPAT, **kw):
    p = _McoParams()
    oracle_lib().mco_default_params(ctypes.byref(p), mode)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def oracle_mesh(ex, ey, ez, lx, ly, lz):
    """The oracle's restatement of load_mesh, returned as MeshArrays."""
    L = oracle_lib()
    m = _McoMesh()
    rc = L.mco_mesh_box(ex, ey, ez, lx, ly, lz, ctypes.byref(m))
    assert rc == 0, rc
    N, F, P = m.cells, m.faces, m.points
    out = MeshArrays(
        ex, ey, ez,
        np.ctypeslib.as_array(m.points_xyz, shape=(P * 3,)).reshape(P, 3).copy(),
        np.ctypeslib.as_array(m.cell_nodes, shape=(N * 8,)).reshape(N, 8).copy(),
        np.ctypeslib.as_array(m.face_cells, shape=(F * 2,)).reshape(F, 2).copy(),
        np.ctypeslib.as_array(m.cell_faces, shape=(N * 6,)).reshape(N, 6).copy(),
        np.ctypeslib.as_array(m.cell_neighbours, shape=(N * 6,)).reshape(N, 6).copy(),
        np.ctypeslib.as_array(m.cell_centers, shape=(N * 3,)).reshape(N, 3).copy(),
        np.array(list(m.boundary_types), dtype=np.uint64))
    L.mco_mesh_free(ctypes.byref(m))
    return out


class Oracle:
    """The C restatement, driven on a mesh given in the reference layout."""

    def __init__(self, mesh, params):
        self.L = oracle_lib()
        self.mesh = mesh
        self._arrays = [np.ascontiguousarray(a) for a in (
            mesh.points.astype(np.float64), mesh.cells.astype(np.uint64), mesh.faces.astype(np.uint64),
            mesh.cell_faces.astype(np.uint64), mesh.cell_neighbours.astype(np.uint64),
            mesh.cell_centers.astype(np.float64))]
        m = _McoMesh()
        m.ex, m.ey, m.ez = mesh.ex, mesh.ey, mesh.ez
        m.cells, m.faces, m.points = mesh.n_cells, mesh.n_faces, mesh.points.shape[0]
        m.points_xyz = self._arrays[0].ctypes.data_as(ctypes.POINTER(c_dbl))
        m.cell_nodes = self._arrays[1].ctypes.data_as(ctypes.POINTER(c_u64))
        m.face_cells = self._arrays[2].ctypes.data_as(ctypes.POINTER(c_u64))
        m.cell_faces = self._arrays[3].ctypes.data_as(ctypes.POINTER(c_u64))
        m.cell_neighbours = self._arrays[4].ctypes.data_as(ctypes.POINTER(c_u64))
        m.cell_centers = self._arrays[5].ctypes.data_as(ctypes.POINTER(c_dbl))
        for i in range(6):
            m.boundary_types[i] = int(mesh.boundary_types[i])
        self._m = m
        self.h = self.L.mco_create(ctypes.byref(m), ctypes.byref(params))
        assert self.h, "mco_create failed"
        self.N = mesh.n_cells
        self.F = mesh.n_faces

    def close(self):
        if self.h:
            self.L.mco_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def field(self, name):
        a = np.zeros(self.N + 6)
        assert self.L.mco_get_field(self.h, FIELDS[name], _ptr(a)) == 0
        return a

    def set_field(self, name, vals):
        a = np.ascontiguousarray(vals, dtype=np.float64)
        assert a.shape == (self.N + 6,)
        assert self.L.mco_set_field(self.h, FIELDS[name], _ptr(a)) == 0

    def grad(self, name):
        a = np.zeros((self.N, 3))
        assert self.L.mco_get_grad(self.h, FIELDS[name], _ptr(a)) == 0
        return a

    def cell_array(self, which):
        a = np.zeros(self.N)
        assert self.L.mco_get_cell_array(self.h, which, _ptr(a)) == 0
        return a

    def face_array(self, which):
        width = {4: 2, 5: 3, 6: 3}.get(which, 1)
        a = np.zeros((self.F, width))
        assert self.L.mco_get_face_array(self.h, which, _ptr(a)) == 0
        return a if width > 1 else a[:, 0]

    def set_sources(self, terms):
        a = np.ascontiguousarray(terms, dtype=np.float64)
        assert a.shape == (self.N, 5)
        self.L.mco_set_sources(self.h, _ptr(a))

    def csr(self, which):
        n, nnz = c_int(), c_int()
        self.L.mco_get_csr(self.h, which, ctypes.byref(n), ctypes.byref(nnz), None, None, None)
        rp = np.zeros(n.value + 1, dtype=np.int32)
        col = np.zeros(nnz.value, dtype=np.int32)
        val = np.zeros(nnz.value)
        self.L.mco_get_csr(self.h, which, ctypes.byref(n), ctypes.byref(nnz), _ptr(rp), _ptr(col), _ptr(val))
        return rp, col, val

    def rhs(self, which):
        a = np.zeros(self.N)
        self.L.mco_get_rhs(self.h, which, _ptr(a))
        return a

    def step(self):
        return self.L.mco_pass(self.h)

    def stage_scalar(self, name):
        return self.L.mco_stage_scalar(self.h, FIELDS[name])

    def stats(self):
        s = _McoStats()
        self.L.mco_get_stats(self.h, ctypes.byref(s))
        return s


_ref_lib = None


def ref_available():
    return os.path.exists(REF_SO)


def ref_lib():
    global _ref_lib
    if _ref_lib is None:
        L = ctypes.CDLL(REF_SO)
        L.mcref_create.argtypes = [c_u64, c_u64, c_u64, c_dbl, c_dbl, c_dbl, c_dbl]
        L.mcref_create.restype = c_vp
        for fn in ("mcref_destroy", "mcref_pass", "mcref_timestep", "mcref_stage_gradients",
                   "mcref_stage_set_up_field", "mcref_stage_calculate_uvw", "mcref_stage_calculate_pressure",
                   "mcref_stage_scalar_temperature"):
            getattr(L, fn).argtypes = [c_vp]
        L.mcref_sizes.argtypes = [c_vp] + [ctypes.POINTER(c_u64)] * 4
        L.mcref_get_mesh.argtypes = [c_vp] + [c_vp] * 7
        L.mcref_set_tolerances.argtypes = [c_dbl, c_dbl, c_int]
        for fn in ("mcref_get_field", "mcref_set_field", "mcref_get_grad", "mcref_get_cell_array",
                   "mcref_get_face_array", "mcref_get_vec"):
            getattr(L, fn).argtypes = [c_vp, c_int, c_vp]
            getattr(L, fn).restype = c_int
        L.mcref_get_csr.argtypes = [c_vp, c_int, ctypes.POINTER(c_int), ctypes.POINTER(c_int), c_vp, c_vp, c_vp]
        L.mcref_first_pressure.argtypes = [c_vp]
        L.mcref_stage_scalar.argtypes = [c_vp, c_int]
        L.mcref_write_flow.argtypes = [c_vp, ctypes.c_char_p, c_int]
        L.mcshim_inject_reset.argtypes = []
        L.mcshim_inject_rank.argtypes = [c_int, ctypes.c_long, c_vp, c_vp, c_int]
        L.mcshim_outbox_count.restype = ctypes.c_long
        L.mcshim_outbox_get.argtypes = [ctypes.c_long, ctypes.POINTER(c_int), ctypes.POINTER(c_int), c_vp]
        L.mcshim_outbox_get.restype = ctypes.c_long
        L.mcref_update_flow_field.argtypes = [c_vp]
        L.mcref_get_particle_terms.argtypes = [c_vp, c_vp]
        L.mcref_stage_scalar.restype = c_int
        L.mcref_timestep_count.argtypes = [c_vp]
        L.mcref_timestep_count.restype = c_u64
        L.mcref_inlet_effective_viscosity.argtypes = [c_vp]
        L.mcref_inlet_effective_viscosity.restype = c_dbl
        L.mcref_last_solve.argtypes = [ctypes.POINTER(c_int), ctypes.POINTER(c_dbl), ctypes.POINTER(c_int)]
        L.mcref_solve_counts.argtypes = [ctypes.POINTER(ctypes.c_long), ctypes.POINTER(ctypes.c_long)]
        _ref_lib = L
    return _ref_lib


class Reference:
    """The reference FlowSolver (one flow rank) behind the harness."""

    def __init__(self, ex, ey, ez, lx, ly, lz, delta=1.0e-5, bcgs_rtol=1e-13, cg_rtol=1e-13, max_iters=100000):
        self.L = ref_lib()
        self.L.mcref_set_tolerances(bcgs_rtol, cg_rtol, max_iters)
        self.h = self.L.mcref_create(ex, ey, ez, lx, ly, lz, delta)
        s = [c_u64() for _ in range(4)]
        self.L.mcref_sizes(self.h, *[ctypes.byref(x) for x in s])
        self.N, self.F, self.P, self.phi_len = [x.value for x in s]
        self.ex, self.ey, self.ez = ex, ey, ez

    def close(self):
        if self.h:
            self.L.mcref_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def mesh(self):
        N, F, P = self.N, self.F, self.P
        pts = np.zeros((P, 3))
        cells = np.zeros((N, 8), dtype=np.uint64)
        faces = np.zeros((F, 2), dtype=np.uint64)
        cf = np.zeros((N, 6), dtype=np.uint64)
        cn = np.zeros((N, 6), dtype=np.uint64)
        cc = np.zeros((N, 3))
        bt = np.zeros(6, dtype=np.uint64)
        self.L.mcref_get_mesh(self.h, _ptr(pts), _ptr(cells), _ptr(faces), _ptr(cf), _ptr(cn), _ptr(cc), _ptr(bt))
        return MeshArrays(self.ex, self.ey, self.ez, pts, cells, faces, cf, cn, cc, bt)

    def field(self, name):
        a = np.zeros(self.phi_len)
        assert self.L.mcref_get_field(self.h, FIELDS[name], _ptr(a)) == 0
        return a

    def set_field(self, name, vals):
        a = np.ascontiguousarray(vals, dtype=np.float64)
        assert a.shape == (self.phi_len,)
        assert self.L.mcref_set_field(self.h, FIELDS[name], _ptr(a)) == 0

    def grad(self, name):
        a = np.zeros((self.N, 3))
        assert self.L.mcref_get_grad(self.h, FIELDS[name], _ptr(a)) == 0
        return a

    def cell_array(self, which):
        a = np.zeros(self.N)
        assert self.L.mcref_get_cell_array(self.h, which, _ptr(a)) == 0
        return a

    def face_array(self, which):
        width = {4: 2, 5: 3, 6: 3}.get(which, 1)
        a = np.zeros((self.F, width))
        assert self.L.mcref_get_face_array(self.h, which, _ptr(a)) == 0
        return a if width > 1 else a[:, 0]

    def csr(self, which):
        n, nnz = c_int(), c_int()
        self.L.mcref_get_csr(self.h, which, ctypes.byref(n), ctypes.byref(nnz), None, None, None)
        rp = np.zeros(n.value + 1, dtype=np.int32)
        col = np.zeros(nnz.value, dtype=np.int32)
        val = np.zeros(nnz.value)
        self.L.mcref_get_csr(self.h, which, ctypes.byref(n), ctypes.byref(nnz), _ptr(rp), _ptr(col), _ptr(val))
        return rp, col, val

    def vec(self, which):
        a = np.zeros(self.N)
        self.L.mcref_get_vec(self.h, which, _ptr(a))
        return a

    def step(self):
        self.L.mcref_pass(self.h)

    def timestep(self):
        self.L.mcref_timestep(self.h)

    def stage_scalar(self, name):
        assert self.L.mcref_stage_scalar(self.h, FIELDS[name]) == 0

    def exchange(self, messages):
        """FlowSolver::update_flow_field with the given messages from particle
        ranks ({rank: (cells, rows[n][5])}, processed in that order).  Returns
        the particle terms [cells][5] and, per rank, the node ids and the
        flow_aos values [n][5] the reference sent back."""
        L = self.L
        L.mcshim_inject_reset()
        keep = []
        for rank, (cells, rows) in messages.items():
            c = np.ascontiguousarray(cells, dtype=np.uint64)
            r = np.ascontiguousarray(rows, dtype=np.float64)
            keep += [c, r]
            L.mcshim_inject_rank(rank, c.shape[0], _ptr(c), _ptr(r), 5)
        L.mcref_update_flow_field(self.h)
        terms = np.zeros((self.N, 5))
        L.mcref_get_particle_terms(self.h, _ptr(terms))
        sent = {}
        for i in range(L.mcshim_outbox_count()):
            d, t = c_int(), c_int()
            nb = L.mcshim_outbox_get(i, ctypes.byref(d), ctypes.byref(t), None)
            buf = np.zeros(nb // 8)
            L.mcshim_outbox_get(i, ctypes.byref(d), ctypes.byref(t), _ptr(buf))
            entry = sent.setdefault(d.value, {})
            entry[t.value] = buf.view(np.uint64) if t.value == 0 else buf.reshape(-1, 5)
        L.mcshim_inject_reset()
        return terms, {r: (e[0], e[1]) for r, e in sent.items()}

    def write_flow(self, prefix, id):
        """The reference's VisitWriter output of the current fields; returns the file name."""
        self.L.mcref_write_flow(self.h, os.fsencode(prefix), int(id))
        return f"{prefix}_flow0_timestep{int(id)}.vtk"

    def inlet_effective_viscosity(self):
        return self.L.mcref_inlet_effective_viscosity(self.h)


def noisy_initial_fields(n_cells, base, seed, amplitude=0.01):
    """Initial interior fields = base * (1 + U(-a, a)) per cell and field, from
    numpy's PCG64 with the given seed (the inlet state plus seeded noise)."""
    rng = np.random.default_rng(seed)
    out = {}
    for name in ("U", "V", "W", "P", "TEM"):
        b = base[name]
        noise = rng.uniform(-amplitude, amplitude, size=n_cells)
        if b == 0.0:
            out[name] = base["U"] * noise  # zero-valued fields: noise of a% of the inlet speed
        else:
            out[name] = b * (1.0 + noise)
    return out
