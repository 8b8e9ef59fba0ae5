"""Generate the golden fixtures under tests/golden/ from the compiled reference.

Needs oracle/_ref (built by `make -C oracle ref` from the reference sources). Every
vector here comes from running the reference's own code: its KAT harness
(oracle/ref_harness.cpp) for function-level vectors and its idx2App CLI for
whole datasets. Inputs are regenerated from seeds; large outputs are stored as
SHA-256 digests.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes as C
import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
REF = os.path.join(ROOT, "oracle", "_ref")

from golden_inputs import (block_cases, brick_cases, finalize_cases, dataset_cases,  # noqa: E402
                           decode_requests, make_block, make_brick, make_dataset_field)


def sha(b: bytes) -> str:
    return hashlib.sha256(b).hexdigest()


def dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def up(a):
    return a.ctypes.data_as(C.POINTER(C.c_ulonglong))


def gen_bricks(ref):
    out = []
    for case in brick_cases():
        b = make_brick(case)
        is2d, valid, level, coarsest = case["is2d"], case["valid"], case["level"], case["coarsest"]
        fwd = b.copy()
        ref.ref_brick_forward(dp(fwd), 1 if is2d else 32, valid[0], valid[1], valid[2], level, coarsest)
        ext = b.copy()
        ref.ref_brick_extrapolate(dp(ext), 1 if is2d else 32, valid[0], valid[1], valid[2])
        inv = fwd.copy()
        ref.ref_brick_inverse(dp(inv), 1 if is2d else 32, level, coarsest)
        out.append(dict(case, forward=sha(fwd.tobytes()), extrapolate=sha(ext.tobytes()),
                        inverse=sha(inv.tobytes()), forward_head=fwd.ravel()[:4].tolist()))
    return out


def gen_blocks(ref):
    out = []
    for case in block_cases():
        vals = make_block(case)
        nd = case["ndims"]
        em = np.zeros(1, np.int32)
        uc = np.zeros(64, np.uint64)
        pb = np.zeros(64, np.int32)
        pn = np.zeros(64, np.int32)
        pbits = np.zeros(64, np.int32)
        pw = np.zeros(256, np.uint64)
        k = ref.ref_block_encode(dp(vals), nd, case["is_f32"], C.c_double(case["tol"]), 1, ip(em), up(uc),
                                 ip(pb), ip(pn), ip(pbits), up(pw))
        nv = 1 << (2 * nd)
        dec = np.zeros(nv)
        if k > 0:
            ref.ref_block_decode(nd, int(em[0]), int(k), ip(pb), up(pw), dp(dec))
        out.append(dict(case, nplanes=int(k), emax=int(em[0]),
                        ucoeffs=sha(uc[:nv].tobytes()), planes=pb[:k].tolist(), nin=pn[:k].tolist(),
                        bits=pbits[:k].tolist(), words=sha(pw[:4 * k].tobytes()),
                        decoded=sha(dec.tobytes())))
    return out


def gen_varints(ref):
    ref.ref_varint_stream.restype = C.c_longlong
    rng = np.random.default_rng(2024)
    out = []
    for t in range(64):
        nvar = int(rng.integers(0, 8))
        nun = int(rng.integers(0, 8))
        v1 = rng.integers(0, 2 ** int(rng.integers(1, 50)), nvar, dtype=np.uint64)
        v2 = rng.integers(0, int(rng.choice([2, 10, 70, 200, 700])), nun).astype(np.uint64)
        vals = np.concatenate([v1, v2]).astype(np.uint64)
        buf = np.zeros(4096, np.uint8)
        nbits = ref.ref_varint_stream(up(vals), nvar, len(vals), buf.ctypes.data_as(C.c_char_p), C.c_longlong(4096))
        out.append(dict(vals=[int(x) for x in vals], n_var=nvar, nbits=int(nbits),
                        bytes=buf[:(nbits + 7) // 8].tobytes().hex()))
    return out


def gen_finalize(ref):
    out = []
    i32 = np.zeros(40 * 16, np.int32)
    u64 = np.zeros(6 * 16, np.uint64)
    strs = C.create_string_buffer(384 * 16)
    nl = np.zeros(1, np.int32)
    g3 = np.zeros(3, np.int32)
    for case in finalize_cases():
        i32[:] = 0
        u64[:] = 0
        C.memset(strs, 0, 384 * 16)
        code = ref.ref_finalize(*case["dims"], 0 if case["dtype"] == "float32" else 1, *case["brick"],
                                case["levels"], C.c_double(1e-3), case["bpc"], case["cpf"], case["fpd"], 1,
                                ip(nl), ip(i32), up(u64), strs, ip(g3))
        rec = dict(case, code=int(code))
        if code == 0:
            L = int(nl[0])
            rec["nlevels"] = L
            rec["group3"] = g3.tolist()
            rec["i32"] = i32[:40 * L].tolist()
            rec["u64"] = [int(x) for x in u64[:6 * L]]
            raw = strs.raw
            rec["strs"] = [[raw[384 * l + 128 * k:384 * l + 128 * (k + 1)].split(b"\0")[0].decode()
                            for k in range(3)] for l in range(L)]
        out.append(rec)
    return out


def gen_masks(ref):
    out = []
    masks = np.zeros(16, np.int32)
    spacing = np.zeros(16 * 8 * 3, np.int32)
    for dims, brick, levels in (((256, 256, 256), (32, 32, 32), 3), ((384, 384, 256), (32, 32, 32), 2),
                                ((512, 512, 1), (32, 32, 1), 3), ((160, 128, 96), (32, 32, 32), 2)):
        for ds in ((0, 0, 0), (1, 1, 1), (2, 2, 2), (3, 3, 3), (0, 1, 2), (2, 0, 1), (1, 0, 0)):
            if brick[2] == 1:
                ds = (ds[0], ds[1], 0)
            masks[:] = 0
            spacing[:] = 0
            code = ref.ref_decode_masks(*dims, *brick, levels, *ds, ip(masks), ip(spacing))
            out.append(dict(dims=dims, brick=brick, levels=levels, ds=ds, code=int(code),
                            masks=masks[:levels].tolist(), spacing=spacing[:levels * 24].tolist()))
    return out


def gen_grids(ref):
    out = []
    o9 = np.zeros(9, np.int32)
    rng = np.random.default_rng(99)
    for t in range(40):
        dims = [int(rng.integers(64, 300)) for _ in range(3)]
        first = [int(rng.integers(0, d)) for d in dims]
        last = [int(rng.integers(f, d)) for f, d in zip(first, dims)]
        if t % 5 == 0:
            first, last = [0, 0, 0], [d - 1 for d in dims]
        ds = [int(rng.integers(0, 4)) for _ in range(3)]
        code = ref.ref_output_grid(*dims, 32, 32, 32, 1, *first, *last, *ds, ip(o9))
        out.append(dict(dims=dims, first=first, last=last, ds=ds, code=int(code), grid=o9.tolist()))
    return out


def gen_datasets():
    """Encode small fields with the reference CLI; keep the files and decoded hashes."""
    app = os.path.join(REF, "idx2App")
    base = os.path.join(HERE, "datasets")
    shutil.rmtree(base, ignore_errors=True)
    os.makedirs(base)
    manifest = []
    for case in dataset_cases():
        f = make_dataset_field(case)
        nx, ny, nz = case["dims"]
        with tempfile.TemporaryDirectory() as tmp:
            raw = os.path.join(tmp, f"{case['name']}-f-[{nx}-{ny}-{nz}]-{case['dtype'].capitalize()}.raw")
            f.tofile(raw)
            args = [app, "--encode", raw, "--num_levels", str(case["levels"]), "--tolerance",
                    repr(case["tol"]), "--out_dir", base]
            if case["brick"][2] == 1:
                args += ["--brick_size", "32", "32", "1"]
            r = subprocess.run(args, capture_output=True, text=True)
            assert r.returncode == 0, r.stdout
            decs = []
            for req in decode_requests(case):
                dargs = [app, "--decode", os.path.join(base, case["name"], "f.idx2"), "--downsampling",
                         *map(str, req["ds"]), "--tolerance", repr(req["tol"]), "--out_dir", tmp,
                         "--out_file", "o.raw"]
                if req.get("first"):
                    dargs += ["--first", *map(str, req["first"]), "--last", *map(str, req["last"])]
                r = subprocess.run(dargs, capture_output=True, text=True)
                assert r.returncode == 0, r.stdout
                data = open(os.path.join(tmp, "o.raw"), "rb").read()
                decs.append(dict(req, sha=sha(data), nbytes=len(data)))
        manifest.append(dict(case, field_sha=sha(f.tobytes()), decodes=decs))
    return manifest


def main():
    ref = C.CDLL(os.path.join(REF, "libidx2_ref_harness.so"))
    golden = dict(
        bricks=gen_bricks(ref),
        blocks=gen_blocks(ref),
        varints=gen_varints(ref),
        finalize=gen_finalize(ref),
        masks=gen_masks(ref),
        grids=gen_grids(ref),
    )
    with open(os.path.join(HERE, "kats.json"), "w") as fp:
        json.dump(golden, fp)
    manifest = gen_datasets()
    with open(os.path.join(HERE, "datasets.json"), "w") as fp:
        json.dump(manifest, fp, indent=1)
    print("golden fixtures written")


if __name__ == "__main__":
    main()
