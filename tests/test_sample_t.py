"""The division-free Hermite sample parameter of the curve kernels
(HermTask::sample_t: t = i / (numPoints - 1) from a per-curve reciprocal and
Markstein's correction) equals IEEE division for every 0 <= i <= n <= 16384,
checked exhaustively by tests/sample_t_check.c (gcc, fma from libm)."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def _run(tmp_path, *defs):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    exe = str(tmp_path / ("check" + "".join(d.strip("-D") for d in defs)))
    subprocess.run([cc, "-O2", "-ffp-contract=off", *defs, os.path.join(HERE, "sample_t_check.c"), "-lm",
                    "-o", exe], check=True)
    return subprocess.run([exe, "16384"], capture_output=True, text=True, timeout=120)


def test_corrected_quotient_equals_ieee_division(tmp_path):
    r = _run(tmp_path)
    assert r.returncode == 0, r.stdout
    assert "134242304 pairs, 0 mismatches" in r.stdout


def test_uncorrected_product_is_caught(tmp_path):
    r = _run(tmp_path, "-DUNCORRECTED")
    assert r.returncode == 1
    assert "mismatch" in r.stdout
