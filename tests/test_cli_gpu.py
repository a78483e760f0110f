"""GPU tests of the command-line program's output paths (pi_b200 --batched): a regular file is
mapped and the device's digits copied straight into it; an output that cannot be mapped (a pipe)
falls back to a buffer and fwrite. Both must hold the reference's 1M digits byte for byte."""
import hashlib
import json
import os
import subprocess

import pytest

from helpers import GOLDEN, pkg

pytestmark = pytest.mark.gpu


def _golden():
    return json.load(open(os.path.join(GOLDEN, "pi_golden.json")))["1000000"]


def test_cli_output_file_is_the_reference_digits(tmp_path):
    out = str(tmp_path / "pi.txt")
    with open(out, "wb") as f:  # an older, longer file is replaced, not overlaid
        f.write(b"x" * 3_000_000)
    subprocess.run([pkg.PI_B200_BIN, "--batched", "--digits", "1000000", "--output", out], check=True,
                   stdout=subprocess.DEVNULL, timeout=600)
    data = open(out, "rb").read()
    g = _golden()
    assert len(data) == g["bytes"] and hashlib.sha256(data).hexdigest() == g["sha256"]


def test_cli_output_to_a_pipe_is_the_reference_digits():
    r = subprocess.run([pkg.PI_B200_BIN, "--batched", "--digits", "1000000", "--output", "/dev/stdout"],
                       stdout=subprocess.PIPE, timeout=600)
    assert r.returncode == 0
    g = _golden()
    data = r.stdout[: g["bytes"]]  # the digits, then the program's own report lines
    assert hashlib.sha256(data).hexdigest() == g["sha256"]
