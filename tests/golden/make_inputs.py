"""Writes the small golden INPUT fields (committed under tests/golden/inputs/)
and the case manifest cases.json.  Run once; the inputs are then fixed bytes,
so the reference binaries (tests/golden/run_reference.sh, on a GPU box) and the
oracle / CUDA path (tests/) all see the same data.

Cases cover: multi-chunk 3-D sinusoid, a partial last chunk with a partial
32-word group, tiny inputs (1, 31, 33 floats, exactly one chunk, one chunk plus
one word), white noise, a power-law Gaussian random field, +-1e6 outliers, a
field of special values (+-0, denormals, NaN, +-Inf, FLT_MAX), all zeros, a
constant, huge magnitudes (lossless region), a ramp, and random float bit
patterns that make chunks incompressible (raw fallback in store, init_send and
resi_send, including the reference's raw-init-chunk quirk).
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from cortado_b200 import fields  # noqa: E402

NOA = {"tag": "noa", "mode": "noa", "store": ["1e-1", "1e-3", "1e-5"], "init": "1e-2", "resi": ["1e-2", "1e-4"]}
ABS = {"tag": "abs", "mode": "abs", "store": ["1e-2", "1e-4", "1e-6"], "init": "1e-3", "resi": ["1e-3", "1e-5"]}
ABS_FINE = {"tag": "abs_fine", "mode": "abs", "store": ["1e-30", "1e-36"], "init": "1e-34", "resi": ["1e-34", "1e-36"]}


def main():
    os.makedirs(os.path.join(HERE, "inputs"), exist_ok=True)
    rng = np.random.Generator(np.random.PCG64(20261203))
    cases = {}

    def put(name, arr, settings):
        arr = np.ascontiguousarray(arr, dtype=np.float32)
        arr.tofile(os.path.join(HERE, "inputs", name + ".f32"))
        cases[name] = settings

    put("sin3d_32", fields.sinusoid((32, 32, 32), 11).numpy(), [NOA, ABS])
    put("sin1d_partial", fields.sinusoid((3 * 4096 + 777,), 12, noise=1e-4).numpy(), [NOA, ABS])
    put("tiny_1", np.array([0.75], np.float32), [ABS])
    put("tiny_31", fields.white(31, 13).numpy(), [NOA, ABS])
    put("tiny_33", fields.white(33, 14).numpy(), [NOA])
    put("one_chunk", fields.sinusoid((16, 16, 16), 15).numpy(), [NOA])
    put("one_chunk_plus1", fields.sinusoid((4097,), 16).numpy(), [NOA])
    put("noise_64k", fields.white(65536, 17).numpy(), [NOA, ABS])
    put("grf_128", fields.grf((128, 128), 18, slope=3.0).numpy(), [NOA, ABS])
    put("outliers_64k", fields.sinusoid((64, 32, 32), 19, outlier_frac=0.01).numpy(), [NOA, ABS])
    sp = rng.standard_normal(4096).astype(np.float32)
    special = np.array([0.0, -0.0, np.nan, np.inf, -np.inf, np.finfo(np.float32).max,
                        -np.finfo(np.float32).max, 1e-45, -1e-45, 1e-40, 1.1754944e-38, -1.1754944e-38],
                       dtype=np.float32)
    sp[rng.choice(4096, size=600, replace=False)] = np.resize(special, 600)
    put("special", sp, [ABS, ABS_FINE])
    put("zeros_40k", np.zeros(10000, np.float32), [ABS])
    put("const", np.full(9000, 3.14159, np.float32), [ABS])
    put("huge", (rng.uniform(1e30, 3e38, 20000) * rng.choice([-1.0, 1.0], 20000)).astype(np.float32), [NOA, ABS])
    put("ramp", np.linspace(-5, 5, 30000, dtype=np.float32), [NOA])
    bits = rng.integers(0, 2**23, 20000, dtype=np.uint32) | (rng.integers(60, 190, 20000, dtype=np.uint32) << 23)
    bits |= rng.integers(0, 2, 20000, dtype=np.uint32) << 31
    put("randbits", bits.view(np.float32), [ABS, ABS_FINE])

    with open(os.path.join(HERE, "cases.json"), "w") as f:
        json.dump(cases, f, indent=1, sort_keys=True)
    print("wrote", len(cases), "cases")


if __name__ == "__main__":
    main()
