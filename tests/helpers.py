"""Shared helpers for the GPU parity tests: numpy <-> device columns."""
import numpy as np
import torch

from yallasql_b200 import _abi as A
from yallasql_b200.ops import DeviceBatch, DeviceColumn

NP_TYPE = {np.dtype(np.int32): A.INT32, np.dtype(np.float32): A.FLOAT32, np.dtype(np.int64): A.INT64,
           np.dtype(np.float64): A.FLOAT64, np.dtype(np.uint8): A.BOOL}


def dev_col(a: np.ndarray, type_: int | None = None, nulls: np.ndarray | None = None) -> DeviceColumn:
    if type_ is None:
        type_ = A.TEXT if a.ndim == 2 else NP_TYPE[a.dtype]
    t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    n = None if nulls is None else torch.from_numpy(np.ascontiguousarray(nulls.astype(np.uint8))).cuda()
    return DeviceColumn(t, type_, n)


def dev_batch(cols: list) -> DeviceBatch:
    out = []
    for c in cols:
        if isinstance(c, tuple):
            out.append(dev_col(*c))
        else:
            out.append(dev_col(c))
    return DeviceBatch(out)


def host(c: DeviceColumn):
    v = c.data.cpu().numpy()
    n = None if c.nulls is None else c.nulls.cpu().numpy().astype(bool)
    return v, n


def oracle_cols(cols: list) -> dict:
    """index -> (values, nulls, type) for oracle.expr_eval."""
    out = {}
    for i, c in enumerate(cols):
        if isinstance(c, tuple):
            a, t = c[0], c[1]
            nl = c[2] if len(c) > 2 else None
        else:
            a, t, nl = c, (A.TEXT if c.ndim == 2 else NP_TYPE[c.dtype]), None
        out[i] = (a, nl, t)
    return out


def rel_close(a, b, tol=1e-6):
    if a is None or b is None:
        return a is None and b is None
    if b == 0:
        return abs(a) <= tol
    return abs(a - b) <= tol * abs(b)
