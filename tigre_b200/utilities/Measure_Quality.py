"""Image quality measures, drop-in for tigre.utilities.Measure_Quality
(Python/tigre/utilities/Measure_Quality.py:26-107): the per-iteration reporting of the
iterative drivers (their Quameasopts keyword).

Measure_Quality(res_prev, res, QualMeasOpts) compares res_prev with res by each of 'RMSE',
'nRMSE', 'CC', 'MSSIM', 'UQI', 'SSD', with the reference's formulas, constants included (its
MSSIM is a single global window with K1 = 0.01, K2 = 0.02 and the dynamic range of res_prev,
scaled by 1/N; nRMSE divides by 1e-5 + sqrt(sum res^2) / N) -- these define the numbers the
reference reports, so they are kept as written.  Inputs may be numpy arrays or CUDA tensors; the
sums run in FP64 where the data are (a device iterate is not copied to the host).
"""
from __future__ import annotations

import numpy as np


def _as64(a):
    if type(a).__module__.startswith("torch"):
        return a.detach().double()
    return np.asarray(a, dtype=np.float64)


def _scalar(v):
    return float(v.item()) if hasattr(v, "item") else float(v)


def Measure_Quality(res_prev, res, QualMeasOpts):  # noqa: N802,N803
    opts = [QualMeasOpts] if isinstance(QualMeasOpts, str) else list(QualMeasOpts)
    a, b = _as64(res_prev), _as64(res)
    n = float(np.prod(a.shape))
    torch_in = not isinstance(a, np.ndarray)
    xp_sum = (lambda t: t.sum()) if torch_in else np.sum
    values = []
    for q in opts:
        if q == "RMSE":
            values.append(_scalar((xp_sum((a - b) ** 2) / n) ** 0.5))
        elif q == "nRMSE":
            rmse = (xp_sum((a - b) ** 2) / n) ** 0.5
            values.append(_scalar(rmse / (0.00001 + xp_sum(b ** 2) ** 0.5 / n)))
        elif q == "CC":
            da, db = a - a.mean(), b - b.mean()
            values.append(_scalar(xp_sum(da * db) / (xp_sum(da * da) * xp_sum(db * db)) ** 0.5))
        elif q == "MSSIM":
            ma, mb = a.mean(), b.mean()
            if _scalar(mb) == 0 and _scalar(ma) == 0:
                raise ValueError("Initializing with 0 matrix not valid")
            k1, k2 = 0.01, 0.02
            d = a.max() - a.min()
            lum = (2 * mb * ma + (k1 * d) ** 2) / (ma ** 2 + mb ** 2 + k1 * d ** 2)
            sa = a.std(unbiased=False) if torch_in else a.std()
            sb = b.std(unbiased=False) if torch_in else b.std()
            con = (2 * sa * sb + (k2 * d) ** 2) / (sa ** 2 + sb ** 2 + k2 * d ** 2)
            delta = xp_sum((a - ma) * (b - mb)) / (n - 1)
            struct = (delta + (k2 * d) ** 2 / 2) / (sa * sb + (k2 * d ** 2) / 2)
            values.append(_scalar(lum * con * struct / n))
        elif q == "UQI":
            ma, mb = a.mean(), b.mean()
            va = a.var(unbiased=False) if torch_in else a.var()
            vb = b.var(unbiased=False) if torch_in else b.var()
            if _scalar(mb) == 0 and _scalar(ma) == 0:
                raise ValueError("Initializing with 0 matrix not valid")
            cova = xp_sum((b - mb) * (a - ma)) / (n - 1)
            values.append(_scalar((2 * cova) / (vb + va) * (2 * mb * ma) / (mb ** 2 + ma ** 2)))
        elif q == "SSD":
            values.append(_scalar(xp_sum((a - b) ** 2)))
    if len(values) == 1:
        return np.array(values[0])
    return np.array(values)


class QualityLog:
    """Quameasopts bookkeeping of a driver: lq[k, it] = measure k between the iterate after
    iteration `it` and the one before it (iterative_recon_alg.py:362-364)."""

    def __init__(self, opts, niter):
        self.opts = None if opts is None else ([opts] if isinstance(opts, str) else list(opts))
        self.lq = None if self.opts is None else np.zeros((len(self.opts), niter))
        self._prev = None

    @property
    def active(self):
        return self.opts is not None

    def before(self, x):
        if self.active:
            self._prev = x.detach().clone() if hasattr(x, "detach") else np.array(x, copy=True)

    def after(self, x, it):
        if self.active:
            self.lq[:, it] = np.atleast_1d(Measure_Quality(x, self._prev, self.opts))

    def errors(self, l2=None):
        """geterrors (iterative_recon_alg.py:406-410): [l2 rows; quality rows]."""
        if l2 is None:
            return self.lq
        l2 = np.asarray(l2, dtype=np.float64).reshape(1, -1)
        return l2 if self.lq is None else np.concatenate((l2, self.lq), axis=0)
