"""Seeded inputs shared by the golden generator and the tests."""
from __future__ import annotations

import numpy as np


def brick_cases():
    rng = np.random.default_rng(101)
    cases = []
    fixed = [(32, 32, 32), (1, 32, 32), (32, 1, 17), (2, 3, 31), (17, 17, 17), (31, 30, 29), (16, 8, 4)]
    for i in range(36):
        is2d = i % 4 == 3
        if i < len(fixed) and not is2d:
            valid = list(fixed[i])
        else:
            valid = [int(rng.integers(1, 33)), int(rng.integers(1, 33)), int(rng.integers(1, 33))]
        if is2d:
            valid[2] = 1
        cases.append(dict(seed=1000 + i, is2d=int(is2d), valid=valid, level=int(rng.integers(0, 3)),
                          coarsest=int(rng.integers(0, 2)), scale=float(10 ** rng.uniform(-4, 4))))
    return cases


def make_brick(case):
    rng = np.random.default_rng(case["seed"])
    nz = 1 if case["is2d"] else 33
    b = np.zeros((nz, 33, 33))
    vx, vy, vz = case["valid"]
    b[:vz, :vy, :vx] = rng.normal(size=(vz, vy, vx)) * case["scale"]
    return b


def block_cases():
    rng = np.random.default_rng(202)
    cases = []
    for i in range(600):
        cases.append(dict(seed=5000 + i, ndims=int(rng.integers(0, 4)), is_f32=int(rng.integers(0, 2)),
                          tol=float(10 ** rng.uniform(-12, -1)), mag=float(10 ** rng.uniform(-8, 6)),
                          kind=int(i % 9)))
    return cases


def make_block(case):
    rng = np.random.default_rng(case["seed"])
    nv = 1 << (2 * case["ndims"])
    v = rng.normal(size=nv) * case["mag"]
    k = case["kind"]
    if k == 1:
        v[:] = 0.0
    elif k == 2:
        v[int(rng.integers(0, nv))] = 5e-310  # denormal
    elif k == 3:
        v = np.abs(v)
    elif k == 4:
        v[:] = case["mag"]
    elif k == 5:
        v = -np.abs(v)
    elif k == 6:
        v[::2] = 0.0
    elif k == 7:
        v = np.round(v)
    return np.ascontiguousarray(v, dtype=np.float64)


def finalize_cases():
    """Shapes of the 512-field uneven set (each axis U{17..300}, 1 in 8 fields 2D with
    z = 1, levels U{1..3}), plus non-default chunk/file parameters."""
    rng = np.random.default_rng(7)
    cases = []
    for i in range(512):
        dims = [int(rng.integers(17, 301)) for _ in range(3)]
        is2d = rng.integers(0, 8) == 0
        if is2d:
            dims[2] = 1
        cases.append(dict(dims=dims, dtype="float32" if i % 2 else "float64",
                          brick=[32, 32, 1] if is2d else [32, 32, 32], levels=int(rng.integers(1, 4)),
                          bpc=4096, cpf=64, fpd=64))
    for i, (bpc, cpf, fpd) in enumerate(((512, 8, 4), (64, 64, 2), (8, 2, 16), (1024, 4096, 4096),
                                         (4096, 64, 64), (100, 64, 64), (4096, 100, 64), (4096, 64, 5000))):
        cases.append(dict(dims=[600, 500, 300], dtype="float32", brick=[32, 32, 32], levels=3, bpc=bpc,
                          cpf=cpf, fpd=fpd))
    return cases


def dataset_cases():
    return [
        dict(name="d64a", dims=(64, 48, 40), dtype="float64", levels=1, tol=1e-3, brick=(32, 32, 32), seed=31),
        dict(name="f32b", dims=(96, 80, 72), dtype="float32", levels=2, tol=1e-3, brick=(32, 32, 32), seed=32),
        dict(name="f32c", dims=(200, 150, 1), dtype="float32", levels=2, tol=1e-3, brick=(32, 32, 1), seed=33),
        dict(name="d64d", dims=(70, 36, 33), dtype="float64", levels=1, tol=1e-5, brick=(32, 32, 32), seed=34),
    ]


def make_dataset_field(case):
    from idx2_b200.synthetic import bumps_field
    nx, ny, nz = case["dims"]
    return bumps_field(nx, ny, nz, seed=case["seed"]).astype(np.float32 if case["dtype"] == "float32"
                                                              else np.float64)


def decode_requests(case):
    nx, ny, nz = case["dims"]
    reqs = [dict(ds=(0, 0, 0), tol=0.0), dict(ds=(1, 1, 0 if nz == 1 else 1), tol=0.0),
            dict(ds=(0, 0, 0), tol=1e-1),
            dict(ds=(0, 0, 0), tol=0.0, first=(nx // 4, ny // 4, nz // 4),
                 last=(3 * nx // 4, 3 * ny // 4, 3 * nz // 4))]
    return reqs
