"""The entry-pass shape table (libssa_b200/csrc/tuning.cpp, written by
libssa_b200/tune.py): the library reads the committed table next to its build,
another file named by SSA_B200_TUNING, or its built-in costs, and reports
which.  CPU only: reading the table touches no device."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_REPORT = "import json, libssa_b200 as L; L.load(); print(json.dumps(L.tuning_report()))"


def _report(env_value: str | None) -> dict:
    env = dict(os.environ)
    env.pop("SSA_B200_TUNING", None)
    if env_value is not None:
        env["SSA_B200_TUNING"] = env_value
    out = subprocess.run([sys.executable, "-c", _REPORT], cwd=ROOT, env=env, capture_output=True, text=True,
                         check=True).stdout
    return json.loads(out.strip().splitlines()[-1])


def test_builtin_table_on_request(built_library):
    r = _report("builtin")
    assert r["source"] == "built-in"
    assert r["version"] == 0
    assert r["last_call"] == []


def test_table_file_is_read(built_library, tmp_path):
    path = tmp_path / "t.tune"
    path.write_text("# a table\nversion 7\ndevice Test Device 1\nqpair 1 20 5 12.5\nfast 4 8 24 3.0\n")
    r = _report(str(path))
    assert r["source"] == str(path)
    assert r["version"] == 7
    assert r["device"] == "Test Device 1"


def test_committed_table_is_the_default(built_library):
    committed = os.path.join(ROOT, "libssa_b200", "tuning", "b200.tune")
    r = _report(None)
    if os.path.exists(committed):
        assert os.path.realpath(r["source"]) == os.path.realpath(committed)
        with open(committed) as f:
            lines = [ln.split() for ln in f if ln.strip() and not ln.startswith("#")]
        version = [int(x[1]) for x in lines if x[0] == "version"]
        assert version and r["version"] == version[0]
        # every database bucket has a measured cost for every query-pair shape
        for kind in ("qpair", "qpair4"):
            qp = {(int(x[1]), int(x[2]), int(x[3])) for x in lines if x[0] == kind}
            assert qp == {(b, R, mb) for b in range(6) for R in (16, 20, 24, 28) for mb in (4, 5)}, kind
        # the fp16x2-maximum variant exists at 4 CTAs per SM only
        qp = {(int(x[1]), int(x[2]), int(x[3])) for x in lines if x[0] == "qpair4h"}
        assert not qp or qp == {(b, R, 4) for b in range(6) for R in (16, 20, 24, 28)}
        # the 8-threads-per-sequence variant exists for the 96-row class only
        qp = {(int(x[1]), int(x[2]), int(x[3])) for x in lines if x[0] == "qpair4g8"}
        assert not qp or qp == {(b, 24, mb) for b in range(6) for mb in (4, 5)}
        # every bucket has a cost for every shape of both single-query kernels
        fast = {(int(x[1]), int(x[2]), int(x[3])) for x in lines if x[0] == "fast"}
        assert fast == {(b, G, R) for b in range(6) for G in (8, 16, 32) for R in (8, 16, 24, 32) if G * R <= 512}
        fast4 = {(int(x[1]), int(x[2]), int(x[3])) for x in lines if x[0] == "fast4"}
        assert fast4 == {(b, G, R) for b in range(6) for G in (4, 8, 16, 32) for R in (8, 16, 24) if G * R <= 512}
    else:
        assert r["source"] == "built-in"


def test_partial_run_keeps_the_other_kernels(tmp_path):
    """python -m libssa_b200.tune --kernels fast re-measures the single-query
    kernels only; the query-pair entries of the existing table are kept."""
    from libssa_b200.tune import kept_entries
    path = tmp_path / "t.tune"
    path.write_text("# c\nversion 3\ndevice X\nqpair 0 16 4 33.5\nqpair4h 1 20 4 26.7  # note\n"
                    "fast 0 8 8 122.2\nfast4 2 4 16 80.0\n")
    assert kept_entries(str(path), ("fast",)) == ["qpair 0 16 4 33.5", "qpair4h 1 20 4 26.7"]
    assert kept_entries(str(path), ("qpair",)) == ["fast 0 8 8 122.2", "fast4 2 4 16 80.0"]
    assert kept_entries(str(tmp_path / "absent.tune"), ("fast",)) == []
