"""ctypes binding of the learned warm start's network (include/espice_mlp.h).

Device arrays are passed as integer pointers (e.g. torch tensors'
data_ptr()); the library owns the network's weights and work buffers.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import lanes

EXPORTS = ["esl_mlp_create", "esl_mlp_destroy", "esl_mlp_last_error", "esl_mlp_set_scaling", "esl_mlp_train",
           "esl_mlp_predict", "esl_mlp_gradients", "esl_mlp_shapes", "esl_mlp_weights", "esl_gemm_bf16",
           "esl_gemm_bf16_bounded"]

GEMM_NO_WAIT = 0xFFFFFFFF  # ESL_GEMM_NO_WAIT: every completion wait runs out at once
MLP_TIMEOUT = 7

f32p = ctypes.POINTER(ctypes.c_float)
i32p = ctypes.POINTER(ctypes.c_int)


def _lib():
    L = lanes.lib()
    if not getattr(L, "_mlp_typed", False):
        L.esl_mlp_last_error.restype = ctypes.c_char_p
        for name in EXPORTS:
            if name != "esl_mlp_last_error":
                getattr(L, name).restype = ctypes.c_int32
        L._mlp_typed = True
    return L


def _fp(a):
    return None if a is None else np.ascontiguousarray(a, np.float32).ctypes.data_as(f32p)


class MlpError(RuntimeError):
    def __init__(self, code, what):
        super().__init__(f"espice_mlp error {code}: {what}")
        self.code = code


def gemm_bf16(d_a, lda, d_b, ldb, M, N, K, d_c, ldc, d_bias=0, d_h=0, ldh=0, act=0, wait_rounds=0):
    """esl_gemm_bf16 (wait_rounds 0), or esl_gemm_bf16_bounded with that
    bound on the tensor-core completion waits."""
    rc = _lib().esl_gemm_bf16_bounded(ctypes.c_void_p(d_a), lda, ctypes.c_void_p(d_b), ldb, M, N, K,
                                      ctypes.c_void_p(d_bias) if d_bias else None, ctypes.c_void_p(d_c), ldc,
                                      ctypes.c_void_p(d_h) if d_h else None, ldh, act,
                                      ctypes.c_uint32(wait_rounds))
    if rc:
        raise MlpError(rc, "esl_gemm_bf16")


class Mlp:
    def __init__(self, n_in, n_hidden, n_layers, n_out, device=0, seed=1):
        self._L = _lib()
        self._m = ctypes.c_void_p()
        rc = self._L.esl_mlp_create(n_in, n_hidden, n_layers, n_out, device, ctypes.c_uint64(seed),
                                    ctypes.byref(self._m))
        if rc:
            self._m = None
            raise MlpError(rc, "esl_mlp_create")
        self.n_in, self.n_out = n_in, n_out

    def _check(self, rc, what):
        if rc:
            msg = self._L.esl_mlp_last_error(self._m)
            raise MlpError(rc, f"{what}: {msg.decode() if msg else ''}")

    def close(self):
        if self._m:
            self._L.esl_mlp_destroy(self._m)
            self._m = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_scaling(self, in_mu=None, in_sig=None, out_mu=None, out_sig=None):
        keep = [np.ascontiguousarray(a, np.float32) if a is not None else None
                for a in (in_mu, in_sig, out_mu, out_sig)]
        self._check(self._L.esl_mlp_set_scaling(self._m, *[_fp(a) for a in keep]), "esl_mlp_set_scaling")

    def train(self, d_x, d_y, n, epochs, batch=256, lr=1e-3, lr_end=0.0, seed=1):
        loss = np.zeros(max(epochs, 1), np.float32)
        self._check(self._L.esl_mlp_train(self._m, ctypes.c_void_p(d_x), ctypes.c_void_p(d_y), ctypes.c_uint32(n),
                                          ctypes.c_uint32(epochs), ctypes.c_uint32(batch), ctypes.c_float(lr),
                                          ctypes.c_float(lr_end), ctypes.c_uint64(seed),
                                          loss.ctypes.data_as(f32p)), "esl_mlp_train")
        return loss[:epochs]

    def predict(self, d_x, n, d_y):
        self._check(self._L.esl_mlp_predict(self._m, ctypes.c_void_p(d_x), ctypes.c_uint32(n),
                                            ctypes.c_void_p(d_y)), "esl_mlp_predict")

    def shapes(self):
        k = (ctypes.c_int * 16)()
        n = (ctypes.c_int * 16)()
        nl = ctypes.c_int(0)
        self._check(self._L.esl_mlp_shapes(self._m, k, n, 16, ctypes.byref(nl)), "esl_mlp_shapes")
        return [(k[i], n[i]) for i in range(nl.value)]

    def _unpack(self, flat):
        out, at = [], 0
        for k, n in self.shapes():
            w = flat[at:at + n * k].reshape(n, k)
            at += n * k
            b = flat[at:at + n]
            at += n
            out.append((w, b))
        return out

    def weights(self):
        total = sum(n * k + n for k, n in self.shapes())
        flat = np.zeros(total, np.float32)
        self._check(self._L.esl_mlp_weights(self._m, flat.ctypes.data_as(f32p)), "esl_mlp_weights")
        return self._unpack(flat)

    def gradients(self, d_x, d_y, n):
        total = sum(nn * k + nn for k, nn in self.shapes())
        flat = np.zeros(total, np.float32)
        loss = ctypes.c_float(0)
        self._check(self._L.esl_mlp_gradients(self._m, ctypes.c_void_p(d_x), ctypes.c_void_p(d_y),
                                              ctypes.c_uint32(n), ctypes.byref(loss), flat.ctypes.data_as(f32p)),
                    "esl_mlp_gradients")
        return loss.value, self._unpack(flat)
