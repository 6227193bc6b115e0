"""The float forms of the quantizers that the kernels use for lossy words
(server quantizer, client quantizer, dequantizer: a power-of-two scale and a
truncating conversion) equal the oracle's integer restatements of the
reference's d_SQ_IABS_4 / d_CQ_IABS_4 / d_iSQ_IABS_4 on every lossy input,
and with the lossless shortcuts (+-(|x| - offs) and |b| + offs) on every
other input: all 2^32 words for two exponents and a stride-97 sweep for the
extremes."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "native", "quant_fast_check.c")


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    from oracle import oracle as O
    lib = O.build()
    exe = str(tmp_path_factory.mktemp("qf") / "quant_fast_check")
    subprocess.check_call(["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-o", exe, SRC, "-lm", "-L",
                           os.path.dirname(lib), "-lcortado_oracle", "-Wl,-rpath," + os.path.dirname(lib)])
    return exe


@pytest.mark.parametrize("eb_e,stride", [(100, 1), (133, 1), (1, 97), (2, 97), (50, 97), (200, 97), (229, 97),
                                         (230, 97)])
def test_float_forms_match_oracle(checker, eb_e, stride):
    r = subprocess.run([checker, str(eb_e), str(stride)], capture_output=True, text=True, timeout=900)
    checked, bad = (int(v) for v in r.stdout.split())
    assert checked > 0
    assert bad == 0 and r.returncode == 0
