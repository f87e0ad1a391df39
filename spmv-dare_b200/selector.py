"""Learned format / tuning selector.

features(): the 10 structural features of a CSR matrix, computed by the GPU kernel behind
spmv_features (the statistics of the reference's generator, artificial-matrix-generator/
artificial_matrix_generation.c:529-570).  MLP: an FP32 10 -> 64 -> 64 -> len(CLASSES)
network whose forward, backward, softmax cross-entropy and Adam steps are the library's own
CUDA kernels (spmv_mlp_*).  Selector: feature normalisation + MLP + the autotuner's class
table; it predicts the class of a matrix from its features and, when its confidence is
below a threshold, falls back to exhaustive autotuning.
"""
from __future__ import annotations

from ctypes import byref, c_float, c_int

import numpy as np

from . import _raise, library, tuning

N_FEATURES = 10
FEATURE_NAMES = ["log2_rows", "log2_nnz", "avg_nnz_per_row", "cov_nnz_per_row", "skew", "avg_bw_scaled",
                 "avg_scatter", "avg_num_neighbours", "cross_row_similarity", "avg_clustering"]


def features(row_ptr, col_ind, m, n):
    """The 10 features of a host CSR matrix (copied to the GPU, computed there)."""
    rp = np.ascontiguousarray(row_ptr, np.int32)
    ci = np.ascontiguousarray(col_ind, np.int32)
    out = np.zeros(N_FEATURES, np.float64)
    st = library().spmv_features(rp.ctypes.data, ci.ctypes.data if ci.size else None, m, n, int(rp[-1]) if m else 0,
                                 out.ctypes.data)
    if st:
        _raise(st)
    return out


def features_device(d_row_ptr, d_col_ind, m, n, nnz, stream=None):
    """The 10 features of a CSR matrix whose arrays are CUDA int32 tensors."""
    out = np.zeros(N_FEATURES, np.float64)
    s = stream.cuda_stream if stream is not None else 0
    st = library().spmv_features_device(d_row_ptr.data_ptr(), d_col_ind.data_ptr() if nnz else None, m, n, nnz,
                                        out.ctypes.data, s or None)
    if st:
        _raise(st)
    return out


def model_inputs(F):
    """Network inputs from raw features: heavy-tailed ones on a log scale."""
    F = np.atleast_2d(np.asarray(F, np.float64)).copy()
    F[:, 2] = np.log(F[:, 2] + 1.0)
    F[:, 4] = np.log1p(np.maximum(F[:, 4], 0.0))
    F[:, 5] = np.log(F[:, 5] + 1e-6)
    F[:, 6] = np.log(F[:, 6] + 1e-6)
    return F


class MLP:
    """FP32 MLP trained and run by the library's CUDA kernels (spmv_mlp_*)."""

    def __init__(self, dims=(N_FEATURES, 64, 64, len(tuning.CLASSES)), seed=0, params=None):
        self.dims = tuple(int(d) for d in dims)
        if params is None:
            params = self.init_params(self.dims, seed)
        params = np.ascontiguousarray(params, np.float32)
        st = c_int(0)
        self._h = library().spmv_mlp_create(*self.dims, params.ctypes.data, byref(st))
        if not self._h:
            _raise(st.value)
        self.num_params = library().spmv_mlp_num_params(self._h)

    @staticmethod
    def init_params(dims, seed):
        """He-uniform weights (bound sqrt(6 / fan_in)), zero biases; seeded PCG64."""
        r = np.random.Generator(np.random.PCG64(seed))
        parts = []
        for l in range(3):
            fan_in, fan_out = dims[l], dims[l + 1]
            bound = np.sqrt(6.0 / fan_in)
            parts.append(r.uniform(-bound, bound, fan_out * fan_in))
            parts.append(np.zeros(fan_out))
        return np.concatenate(parts).astype(np.float32)

    def _get(self, which):
        out = np.empty(self.num_params, np.float32)
        st = library().spmv_mlp_get(self._h, which, out.ctypes.data)
        if st:
            _raise(st)
        return out

    def params(self):
        return self._get(0)

    def grads(self):
        return self._get(1)

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        if p.size != self.num_params:
            raise ValueError(f"expected {self.num_params} parameters")
        st = library().spmv_mlp_set(self._h, p.ctypes.data)
        if st:
            _raise(st)

    def loss_grad(self, xd, labels_d, stream=None):
        """Mean softmax cross-entropy of a [B, in] float32 CUDA batch; gradients kept."""
        loss = c_float(0.0)
        s = stream.cuda_stream if stream is not None else None
        st = library().spmv_mlp_loss_grad(self._h, xd.data_ptr(), labels_d.data_ptr(), xd.shape[0], byref(loss), s)
        if st:
            _raise(st)
        return loss.value

    def adam_step(self, lr, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0, stream=None):
        s = stream.cuda_stream if stream is not None else None
        st = library().spmv_mlp_adam_step(self._h, lr, beta1, beta2, eps, weight_decay, s)
        if st:
            _raise(st)

    def logits(self, xd, out=None, stream=None):
        import torch

        if out is None:
            out = torch.empty((xd.shape[0], self.dims[3]), dtype=torch.float32, device=xd.device)
        s = stream.cuda_stream if stream is not None else None
        st = library().spmv_mlp_forward(self._h, xd.data_ptr(), xd.shape[0], out.data_ptr(), s)
        if st:
            _raise(st)
        return out

    def logits_host(self, X):
        """Logits of a host float32 batch [B, in] (copied in and out by the library)."""
        X = np.ascontiguousarray(X, np.float32)
        out = np.empty((X.shape[0], self.dims[3]), np.float32)
        st = library().spmv_mlp_forward_host(self._h, X.ctypes.data, X.shape[0], out.ctypes.data)
        if st:
            _raise(st)
        return out

    def destroy(self):
        if getattr(self, "_h", None):
            library().spmv_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


class Selector:
    """Feature normalisation + MLP over the autotuner's classes."""

    def __init__(self, mlp, mean, std):
        self.mlp = mlp
        self.mean = np.asarray(mean, np.float64)
        self.std = np.asarray(std, np.float64)

    @classmethod
    def train(cls, F, labels, epochs=400, batch=128, lr=3e-3, weight_decay=1e-4, seed=0, hidden=64, log=None):
        """Trains on raw features F [N, 10] and best-class labels [N] with minibatch Adam on the GPU."""
        import torch

        X = model_inputs(F)
        mean, std = X.mean(0), X.std(0)
        std[std < 1e-12] = 1.0
        Z = torch.from_numpy(((X - mean) / std).astype(np.float32)).cuda()
        y = torch.from_numpy(np.asarray(labels, np.int32)).cuda()
        mlp = MLP((N_FEATURES, hidden, hidden, len(tuning.CLASSES)), seed=seed)
        r = np.random.Generator(np.random.PCG64(seed + 1))
        N = Z.shape[0]
        losses = []
        for ep in range(epochs):
            perm = torch.from_numpy(r.permutation(N)).cuda()
            tot = 0.0
            for b0 in range(0, N, batch):
                idx = perm[b0:b0 + batch]
                loss = mlp.loss_grad(Z[idx].contiguous(), y[idx].contiguous())
                mlp.adam_step(lr, weight_decay=weight_decay)
                tot += loss * idx.numel()
            losses.append(tot / N)
            if log and (ep % 50 == 0 or ep == epochs - 1):
                log(f"epoch {ep} loss {losses[-1]:.4f}")
        sel = cls(mlp, mean, std)
        sel.losses = losses
        return sel

    def proba(self, F):
        Z = ((model_inputs(F) - self.mean) / self.std).astype(np.float32)
        z = self.mlp.logits_host(Z).astype(np.float64)
        z -= z.max(axis=1, keepdims=True)
        e = np.exp(z)
        return e / e.sum(axis=1, keepdims=True)

    def predict(self, F):
        return np.argmax(self.proba(F), axis=1)

    def choose(self, sb, row_ptr, col_ind, values, m, n, fallback_threshold=0.0, timer=None):
        """(class index, how): the MLP's class from the GPU features, or the exhaustive
        autotuner's when the MLP's top probability is below fallback_threshold."""
        p = self.proba(features(row_ptr, col_ind, m, n))[0]
        k = int(np.argmax(p))
        if p[k] >= fallback_threshold:
            return k, "mlp"
        if timer is None:
            import torch

            timer = tuning.Timer(torch, "cuda")
        _, best, _ = tuning.exhaustive(sb, timer, row_ptr, col_ind, values, m, n)
        return best, "exhaustive"

    def save(self, path):
        np.savez(path, params=self.mlp.params(), dims=np.array(self.mlp.dims), mean=self.mean, std=self.std)

    @classmethod
    def load(cls, path):
        with np.load(path) as z:
            mlp = MLP(tuple(z["dims"].tolist()), params=z["params"])
            return cls(mlp, z["mean"], z["std"])
