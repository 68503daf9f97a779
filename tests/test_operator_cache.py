"""On-disk operator cache (KFMM_OPERATOR_CACHE): the first process computes
and stores the NP's operators, later processes load them; the loaded
matrices are bit-identical to computed ones; a damaged file is ignored and
replaced.  Each step runs in a fresh process (the in-process cache would
otherwise answer)."""
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SCRIPT = """
import sys, time, numpy as np
sys.path.insert(0, {root!r})
import __graft_entry__ as g
K = g.load_package()
t = time.time()
ops = K.operators({np_})
np.savez(sys.argv[1], **ops)
print(time.time() - t)
"""


def _run(tmp, np_, out, cache):
    env = dict(os.environ)
    env.pop("KFMM_OPERATOR_CACHE", None)
    if cache:
        env["KFMM_OPERATOR_CACHE"] = str(cache)
    r = subprocess.run([sys.executable, "-c", SCRIPT.format(root=ROOT, np_=np_), str(out)],
                       env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-800:]
    return dict(np.load(out))


def test_operator_cache_round_trip(tmp_path):
    np_ = 4
    cache = tmp_path / "ops"
    cache.mkdir()
    ref = _run(tmp_path, np_, tmp_path / "ref.npz", None)
    first = _run(tmp_path, np_, tmp_path / "a.npz", cache)
    path = cache / f"kifmm_operators_np{np_}.bin"
    assert path.exists()
    second = _run(tmp_path, np_, tmp_path / "b.npz", cache)
    for k in ref:
        assert np.array_equal(ref[k], first[k]) and np.array_equal(ref[k], second[k]), k
    # damage one payload byte: ignored, recomputed, rewritten
    raw = bytearray(path.read_bytes())
    raw[100] ^= 0xFF
    path.write_bytes(bytes(raw))
    third = _run(tmp_path, np_, tmp_path / "c.npz", cache)
    for k in ref:
        assert np.array_equal(ref[k], third[k]), k
    assert path.read_bytes() != bytes(raw)
    # a truncated file is ignored too
    path.write_bytes(bytes(raw[:64]))
    fourth = _run(tmp_path, np_, tmp_path / "d.npz", cache)
    for k in ref:
        assert np.array_equal(ref[k], fourth[k]), k
