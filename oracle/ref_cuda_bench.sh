#!/usr/bin/env bash
# Times the reference's own CUDA build (oracle/_ref, built by oracle/ref.mk) on
# the benchmark field: the 512^3 sinusoid + noise + 0.1% +-1e6 outliers field
# (written to a temporary file by cortado_b200.fields), NOA flow
# store 1e-4 / init 1e-2 / residual 1e-2 -> 1e-4 and ABS flow store 1e-6 /
# init 1e-3 / residual 1e-3 -> 1e-5, each op median of 10 runs (-r 10) as the
# reference's benchmark binaries report it (their timer includes the wrapper's
# cudaMalloc/cudaFree of the carry array).  Needs a GPU.
# Usage: oracle/ref_cuda_bench.sh [outdir]
set -u
HERE="$(cd "$(dirname "$0")" && pwd)"
ROOT="$(cd "$HERE/.." && pwd)"
OUT="${1:-${TMPDIR:-/tmp}/cortado_refbench}"
mkdir -p "$OUT"
F="${TMPDIR:-/tmp}/cortado_field_512.f32"
python3 -c "
import sys; sys.path.insert(0, '$ROOT')
from cortado_b200 import fields
fields.sinusoid((512, 512, 512), 2, outlier_frac=1e-3, device='cuda').reshape(-1).cpu().numpy().tofile('$F')
"
R="$HERE/_ref"
"$R/store_bench" "$F" 1e-4 -r 10 > "$OUT/noa_store.log" 2>&1
"$R/init_bench" "$F" 1e-4 1e-2 -r 10 > "$OUT/noa_init.log" 2>&1
"$R/resi_bench" "$F" 1e-4 1e-2 1e-4 -r 10 > "$OUT/noa_resi.log" 2>&1
"$R/store_bench" "$F" 1e-6 -a -r 10 > "$OUT/abs_store.log" 2>&1
"$R/init_bench" "$F" 1e-6 1e-3 -a -r 10 > "$OUT/abs_init.log" 2>&1
"$R/resi_bench" "$F" 1e-6 1e-3 1e-5 -a -r 10 > "$OUT/abs_resi.log" 2>&1
rm -f "$F"
grep -H -E "runtime|throughput|encoded size" "$OUT"/*.log
