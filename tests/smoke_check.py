"""One small encode on cuda:0 through the C ABI, checked against the oracle's CPU
brick coder driving the same host packer (structural file parity)."""
import os
import tempfile

import numpy as np


def run_smoke():
    import idx2_b200
    from idx2_b200.synthetic import bumps_field
    from idx2_files import compare_dirs
    from oracle_tools import oracle_encode

    with tempfile.TemporaryDirectory() as tmp:
        for dims, dtype, levels, tol in (((64, 48, 40), "float32", 1, 1e-3),
                                         ((128, 100, 70), "float64", 2, 1e-4)):
            f = bumps_field(*dims, seed=11).astype(dtype)
            raw = os.path.join(tmp, f"in-{dtype}.raw")
            f.tofile(raw)
            out_o = os.path.join(tmp, f"oracle-{dtype}")
            rc, err = oracle_encode(raw, dims, dtype, levels, tol, out_o)
            assert rc == 0, err
            out_g = os.path.join(tmp, f"gpu-{dtype}")
            info = idx2_b200.encode(f, out_dir=out_g, name="kat", field_name="f",
                                    num_levels=levels, tolerance=tol)
            assert info.kernel_launches >= 1
            diffs = compare_dirs(os.path.join(out_o, "kat"), os.path.join(out_g, "kat"))
            assert diffs == [], f"GPU encode differs from the oracle: {diffs[:3]}"
    print("smoke ok")


if __name__ == "__main__":
    run_smoke()
