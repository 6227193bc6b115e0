#!/usr/bin/env bash
# Runs the reference's own CLI binaries (built from its sources into
# oracle/_ref by oracle/ref.mk) over every case in tests/golden/cases.json and
# writes their streams, decoded files and logs under $1 (default: a new
# temporary directory, printed at the end).  Needs a GPU.  tests/golden/collect.py then turns the
# outputs into tests/golden/reference_outputs.json (hashes + sizes).
#
# Usage: tests/golden/run_reference.sh [outdir] [extra_input.f32 ...]
set -u
HERE="$(cd "$(dirname "$0")" && pwd)"
ROOT="$(cd "$HERE/../.." && pwd)"
REF="$ROOT/oracle/_ref"
OUT="${1:-$(mktemp -d "${TMPDIR:-/tmp}/cortado_golden.XXXXXX")}"
shift || true
mkdir -p "$OUT"
python3 - "$HERE/cases.json" "$@" > "$OUT/plan.txt" << 'PY'
import json, sys, os
cases = json.load(open(sys.argv[1]))
here = os.path.dirname(sys.argv[1])
for name, settings in sorted(cases.items()):
    for s in settings:
        print(name, os.path.join(here, "inputs", name + ".f32"), s["tag"], s["mode"], " ".join(s["store"]), s["init"], " ".join(s["resi"]), sep="|")
for extra in sys.argv[2:]:
    name = os.path.splitext(os.path.basename(extra))[0]
    print(name, extra, "noa", "noa", "1e-1 1e-3 1e-5", "1e-2", "1e-2 1e-4", sep="|")
PY
while IFS='|' read -r name input tag mode stor init resi; do
  d="$OUT/$name/$tag"
  mkdir -p "$d"
  flag=""; [ "$mode" = "abs" ] && flag="-a"
  set -- $resi; src="$1"; dst="$2"
  "$REF/store" "$input" $stor $flag -o "$d/stor" > "$d/store.log" 2>&1; echo "store $?" > "$d/rc.txt"
  "$REF/init_send" "$d/stor" "$init" $flag -c "$d/init.bin" > "$d/init_send.log" 2>&1; echo "init_send $?" >> "$d/rc.txt"
  "$REF/init_recv" "$d/init.bin" -d "$d/init_dec.f32" > "$d/init_recv.log" 2>&1; echo "init_recv $?" >> "$d/rc.txt"
  "$REF/resi_send" "$d/stor" "$src" "$dst" $flag -c "$d/resi.bin" > "$d/resi_send.log" 2>&1; echo "resi_send $?" >> "$d/rc.txt"
  "$REF/resi_recv" "$d/init_dec.f32" "$d/resi.bin" -d "$d/resi_dec.f32" > "$d/resi_recv.log" 2>&1; echo "resi_recv $?" >> "$d/rc.txt"
  # determinism probe: repeat the decoders on identical inputs
  for k in 1 2 3 4; do
    "$REF/resi_recv" "$d/init_dec.f32" "$d/resi.bin" -d "$d/resi_dec.rep.f32" > /dev/null 2>&1
    sha256sum "$d/resi_dec.rep.f32" | cut -d' ' -f1 >> "$d/resi_recv_repeat.txt"
    "$REF/init_recv" "$d/init.bin" -d "$d/init_dec.rep.f32" > /dev/null 2>&1
    sha256sum "$d/init_dec.rep.f32" | cut -d' ' -f1 >> "$d/init_recv_repeat.txt"
  done
  rm -f "$d/resi_dec.rep.f32" "$d/init_dec.rep.f32"
  "$REF/store_bench" "$input" $stor $flag -v > "$d/store_bench.log" 2>&1; echo "store_bench $?" >> "$d/rc.txt"
  lastst="${stor##* }"
  "$REF/init_bench" "$input" "$lastst" "$init" $flag -v > "$d/init_bench.log" 2>&1; echo "init_bench $?" >> "$d/rc.txt"
  "$REF/resi_bench" "$input" "$lastst" "$src" "$dst" $flag -v > "$d/resi_bench.log" 2>&1; echo "resi_bench $?" >> "$d/rc.txt"
done < "$OUT/plan.txt"
echo "reference golden run complete: $OUT"
