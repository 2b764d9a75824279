"""Python mirror of the learned pressure-guess C ABI (include/minicombust_gnn.h).

Sample arrays are CUDA tensors (float32, one value per cell in the mesh's
own numbering); torch only supplies device memory here.  The network, its
forward and backward passes and Adam all run in the library's kernels.
"""
import ctypes
from ctypes import c_double, c_float, c_int, c_uint64, c_void_p

import numpy as np

from . import flow


class Sample(ctypes.Structure):
    _fields_ = [("rhs", c_void_p), ("diag", c_void_p), ("prev", c_void_p), ("target", c_void_p)]


_SIGNATURES = {
    "mc_gnn_param_count": (c_int, []),
    "mc_gnn_create": (c_int, [c_int, c_uint64, ctypes.POINTER(c_void_p)]),
    "mc_gnn_destroy": (c_int, [c_void_p]),
    "mc_gnn_set_params": (c_int, [c_void_p, c_void_p, c_int]),
    "mc_gnn_get_params": (c_int, [c_void_p, c_void_p, c_int]),
    "mc_gnn_graph_create": (c_int, [c_void_p, ctypes.POINTER(flow.MeshView), ctypes.POINTER(c_void_p)]),
    "mc_gnn_graph_destroy": (c_int, [c_void_p]),
    "mc_gnn_graph_export": (c_int, [c_void_p, ctypes.POINTER(c_int), c_void_p, c_void_p, c_void_p]),
    "mc_gnn_predict": (c_int, [c_void_p, c_void_p, ctypes.POINTER(Sample), c_void_p, c_void_p]),
    "mc_gnn_loss_grad": (c_int, [c_void_p, c_void_p, c_int, ctypes.POINTER(Sample), ctypes.POINTER(c_double),
                                 c_void_p]),
    "mc_gnn_adam_step": (c_int, [c_void_p, c_float]),
    "mc_gnn_train_step": (c_int, [c_void_p, c_void_p, c_int, ctypes.POINTER(Sample), c_float,
                                  ctypes.POINTER(c_double)]),
}

_bound = False


def library():
    global _bound
    L = flow.library()
    if not _bound:
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _bound = True
    return L


def param_count():
    return library().mc_gnn_param_count()


def _dptr(t):
    if t is None:
        return None
    assert t.is_cuda and t.is_contiguous(), "sample arrays must be contiguous CUDA tensors"
    return c_void_p(t.data_ptr())


def _sample(rhs, diag, prev=None, target=None):
    return Sample(_dptr(rhs), _dptr(diag), _dptr(prev), _dptr(target))


class Graph:
    """The cell-face graph of a flow.Mesh on the network's device."""

    def __init__(self, net, mesh):
        self.L = library()
        self._mv = mesh.view()
        h = c_void_p()
        flow._check(self.L.mc_gnn_graph_create(net.h, ctypes.byref(self._mv), ctypes.byref(h)),
                    what="mc_gnn_graph_create")
        self.h = h
        self.n = mesh.n_cells

    def export(self):
        n = c_int()
        col = np.empty((6, self.n), dtype=np.int32)
        edge = np.empty((6, self.n), dtype=np.uint32)
        vhat = np.empty(self.n, dtype=np.float32)
        flow._check(self.L.mc_gnn_graph_export(self.h, ctypes.byref(n), col.ctypes.data_as(c_void_p),
                                               edge.ctypes.data_as(c_void_p), vhat.ctypes.data_as(c_void_p)),
                    what="mc_gnn_graph_export")
        return col, edge, vhat

    def close(self):
        if self.h:
            self.L.mc_gnn_graph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GuessNet:
    """The learned pressure-correction guess: parameters, Adam state and kernels."""

    def __init__(self, device=0, seed=0):
        self.L = library()
        h = c_void_p()
        flow._check(self.L.mc_gnn_create(device, seed, ctypes.byref(h)), what="mc_gnn_create")
        self.h = h
        self.nparam = self.L.mc_gnn_param_count()

    def params(self):
        p = np.empty(self.nparam, dtype=np.float32)
        flow._check(self.L.mc_gnn_get_params(self.h, p.ctypes.data_as(c_void_p), self.nparam), what="get_params")
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        flow._check(self.L.mc_gnn_set_params(self.h, p.ctypes.data_as(c_void_p), len(p)), what="set_params")

    def graph(self, mesh):
        return Graph(self, mesh)

    def predict(self, graph, rhs, diag, prev=None, y=None, x0=None):
        s = _sample(rhs, diag, prev)
        flow._check(self.L.mc_gnn_predict(self.h, graph.h, ctypes.byref(s), _dptr(y), _dptr(x0)), what="predict")

    def loss_grad(self, graph, samples, want_grad=True):
        """samples: list of (rhs, diag, prev, target) CUDA tensors.  Returns (loss, grad or None)."""
        arr = (Sample * len(samples))(*[_sample(*s) for s in samples])
        loss = c_double()
        g = np.empty(self.nparam, dtype=np.float32) if want_grad else None
        flow._check(self.L.mc_gnn_loss_grad(self.h, graph.h, len(samples), arr, ctypes.byref(loss),
                                            g.ctypes.data_as(c_void_p) if g is not None else None),
                    what="loss_grad")
        return loss.value, g

    def train_step(self, graph, samples, lr):
        arr = (Sample * len(samples))(*[_sample(*s) for s in samples])
        loss = c_double()
        flow._check(self.L.mc_gnn_train_step(self.h, graph.h, len(samples), arr, lr, ctypes.byref(loss)),
                    what="train_step")
        return loss.value

    def close(self):
        if self.h:
            self.L.mc_gnn_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
