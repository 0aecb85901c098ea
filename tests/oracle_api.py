"""ctypes access to the CPU oracle (test infrastructure)."""
import ctypes as C

import numpy as np

UINT64_MAX = (1 << 64) - 1


class OParams(C.Structure):
    _fields_ = [("L", C.c_int), ("Imax", C.c_int), ("Tmax", C.c_uint64), ("thres", C.c_double),
                ("alpha", C.c_double * 150)]


class OStats(C.Structure):
    _fields_ = [("iterations", C.c_double), ("ng", C.c_uint64), ("ng_p", C.c_uint64),
                ("converged", C.c_int), ("phases", C.c_int)]


class OLine(C.Structure):
    _fields_ = [("lapp", C.c_double * 16), ("le", C.c_double * 16), ("n_guess", C.c_uint64),
                ("cur_l", C.c_int), ("pnl", C.c_double)]


_DP = np.ctypeslib.ndpointer(np.float64, flags="C")
_U8 = np.ctypeslib.ndpointer(np.uint8, flags="C")


class Oracle:
    def __init__(self, path):
        self.lib = lib = C.CDLL(path)
        lib.sgo_default_params.argtypes = [C.POINTER(OParams)]
        lib.sgo_decode.argtypes = [_DP, C.c_size_t, C.POINTER(OParams), _U8, _DP, C.POINTER(OStats)]
        lib.sgo_bitso.argtypes = [_DP, C.c_int, C.c_uint64, C.c_double, C.POINTER(OLine)]
        lib.sgo_exp.restype = lib.sgo_log.restype = C.c_double
        lib.sgo_exp.argtypes = lib.sgo_log.argtypes = [C.c_double]
        lib.sgo_pattern_order.restype = C.c_size_t
        lib.sgo_pattern_order.argtypes = [C.c_int32, np.ctypeslib.ndpointer(np.uint32, flags="C"), C.c_size_t]
        lib.sgo_encode.argtypes = [_U8, _U8]
        lib.sgo_sigma.restype = C.c_double
        lib.sgo_sigma.argtypes = [C.c_double]
        lib.sgo_early_termination.argtypes = [_DP]

    def params(self, L=3, Imax=30, Tmax=UINT64_MAX, thres=1.0 - 1e-5, alpha=None):
        p = OParams()
        self.lib.sgo_default_params(C.byref(p))
        p.L, p.Imax, p.Tmax, p.thres = L, Imax, Tmax, thres
        if alpha is not None:
            for i, a in enumerate(alpha[:150]):
                p.alpha[i] = a
        return p

    def decode(self, llr, **kw):
        llr = np.ascontiguousarray(llr, dtype=np.float64).reshape(-1, 4096)
        n = llr.shape[0]
        p = self.params(**kw)
        bits = np.zeros(n * 64, np.uint8)
        lapp = np.zeros(n * 4096)
        st = (OStats * n)()
        self.lib.sgo_decode(llr.ravel(), n, C.byref(p), bits, lapp, st)
        stats = [(s.iterations, s.ng, s.ng_p, s.converged, s.phases) for s in st]
        return bits.reshape(n, 64), stats, lapp.reshape(n, 4096)

    def bitso(self, lines, L=3, Tmax=UINT64_MAX, thres=1.0 - 1e-5):
        lines = np.ascontiguousarray(lines, dtype=np.float64).reshape(-1, 16)
        n = lines.shape[0]
        lapp = np.zeros((n, 16))
        le = np.zeros((n, 16))
        ng = np.zeros(n, np.int64)
        nc = np.zeros(n, np.int64)
        for i in range(n):
            o = OLine()
            self.lib.sgo_bitso(np.ascontiguousarray(lines[i]), L, Tmax, thres, C.byref(o))
            lapp[i], le[i], ng[i], nc[i] = o.lapp, o.le, o.n_guess, o.cur_l
        return lapp, le, ng, nc


def twin_decode_one(args):
    """Pool worker: twin oracle decode of one cube with keyword params."""
    path, llr, kw = args
    bits, stats, lapp = Oracle(path).decode(llr, **kw)
    return bits[0], stats[0], lapp[0]


def adjoint(lib_path, llr, code_bits, loss_mode=0, **kw):
    """C FP64 adjoint of one codeword: (loss, grad_alpha[3*Imax], grad_llr[4096])."""
    o = Oracle(lib_path)
    lib = o.lib
    lib.sgo_decode_adjoint.argtypes = [_DP, C.POINTER(OParams), _U8, C.c_int, C.POINTER(C.c_double), _DP, _DP]
    p = o.params(**kw)
    ga = np.zeros(3 * p.Imax)
    gl = np.zeros(4096)
    loss = C.c_double()
    lib.sgo_decode_adjoint(np.ascontiguousarray(llr, dtype=np.float64), C.byref(p),
                           np.ascontiguousarray(code_bits, dtype=np.uint8), int(loss_mode), C.byref(loss), ga, gl)
    return loss.value, ga, gl


def forward_loss(lib_path, llr, code_bits, **kw):
    o = Oracle(lib_path)
    lib = o.lib
    lib.sgo_decode_loss.restype = C.c_double
    lib.sgo_decode_loss.argtypes = [_DP, C.POINTER(OParams), _U8]
    p = o.params(**kw)
    return lib.sgo_decode_loss(np.ascontiguousarray(llr, dtype=np.float64), C.byref(p),
                               np.ascontiguousarray(code_bits, dtype=np.uint8))
