"""Schedule autotuner: the host-side table (candidates, built-in rules, batch
classes, set/get, listing, save/load).  No GPU: these entry points touch no
device."""
import os

import pytest

from tests.test_abi_cpu import _lib


@pytest.fixture()
def tuner():
    o, _ = _lib()
    t = o.Tuner()
    t.set_sms(148)
    yield o, t
    t.close()


def test_candidates(tuner):
    o, t = tuner
    assert t.candidates("lu", 882) == [0, 1, 2]
    assert t.candidates("lu", 200) == [0, 1]
    assert t.candidates("product", 98) == [0, 1, 2]
    assert t.candidates("schur", 242) == [64, 96, 128, 192]
    assert t.candidates("schur", 882) == [64]  # large matrices: multishift phase dominates
    assert t.candidates("schur", 40) == [64]   # below the crossover: single-shift only
    with pytest.raises(o.RcwaError):
        t.candidates(7, 100)


def test_default_rules(tuner):
    _, t = tuner
    # LU: one CTA per matrix for n <= 128 or >= 4 waves of matrices, else
    # 128-column blocks from n = 256 on, panels below
    assert t.default("lu", 882, 148) == 2
    assert t.default("lu", 882, 591) == 2
    assert t.default("lu", 200, 148) == 1
    assert t.default("lu", 882, 592) == 0
    assert t.default("lu", 128, 10) == 0
    assert t.default("schur", 882, 740) == 64
    assert t.default("schur", 98, 200) == 128   # small matrices: single-shift kernel
    assert t.default("schur", 40, 200) == 64    # the only candidate below 64 rows
    assert t.default("product", 882, 148) == 0
    t.set_sms(100)
    assert t.default("lu", 882, 400) == 0


def test_set_get_batch_classes(tuner):
    _, t = tuner
    t.set("lu", 882, 296, 0)                 # 2 waves
    assert t.get("lu", 882, 290) == 0        # same class
    assert t.get("lu", 882, 148) is None     # 1 wave
    assert t.get("lu", 880, 296) is None     # other order
    t.set("schur", 450, 600, 128)            # 5 waves -> class 4 (4..7 waves)
    assert t.get("schur", 450, 1000) == 128
    assert t.get("schur", 450, 1200) is None  # 9 waves -> class 8
    t.set("lu", 882, 296, 1)                 # replaces
    assert t.get("lu", 882, 296) == 1
    ents = t.entries()
    assert [(e["op"], e["n"], e["batch_class"], e["choice"]) for e in ents] == [("lu", 882, 2, 1),
                                                                                ("schur", 450, 4, 128)]


def test_invalid_choices_rejected(tuner):
    o, t = tuner
    with pytest.raises(o.RcwaError):
        t.set("schur", 450, 10, 80)
    with pytest.raises(o.RcwaError):
        t.set("lu", 882, 10, 3)
    with pytest.raises(o.RcwaError):
        t.set("lu", 200, 10, 2)   # 128-column blocks need n >= 256
    with pytest.raises(o.RcwaError):
        t.set("schur", 40, 10, 96)
    with pytest.raises(o.RcwaError):
        t.set("lu", 0, 10, 0)
    assert t.entries() == []


def test_save_load_round_trip(tuner, tmp_path):
    o, t = tuner
    t.set("lu", 882, 296, 0)
    t.set("schur", 242, 20, 96)
    t.set("product", 98, 5000, 1)
    path = os.path.join(tmp_path, "sched.txt")
    t.save(path)
    u = o.Tuner()
    u.set_sms(148)
    u.load(path)
    assert u.entries() == t.entries()
    # a hand-written table with timings; entries replace those with the same key
    with open(path, "w") as f:
        f.write("# comment\nschur 242 1 128 64 10.5 96 9.25 128 8.0 192 8.5\n")
    u.load(path)
    e = [x for x in u.entries() if x["op"] == "schur"][0]
    assert e["choice"] == 128 and e["ms"] == {64: 10.5, 96: 9.25, 128: 8.0, 192: 8.5}
    assert len(u.entries()) == 3
    u.close()


def test_load_rejects_bad_files_whole(tuner, tmp_path):
    o, t = tuner
    path = os.path.join(tmp_path, "bad.txt")
    for body in ["lu 882 2 1\nschur 450 1 80\n",      # choice not a candidate
                 "lu 882 5 1\n",                      # batch class 5 does not exist
                 "gemm 882 1 0\n",                    # unknown decision
                 "lu 882\n"]:                         # truncated
        with open(path, "w") as f:
            f.write(body)
        with pytest.raises(o.RcwaError):
            t.load(path)
        assert t.entries() == []
    with pytest.raises(o.RcwaError):
        t.load(os.path.join(tmp_path, "missing.txt"))


def test_schedule_table_from_plain_c(tmp_path):
    # the same table calls from a C program linked against the library
    import subprocess
    from tests.test_abi_cpu import ROOT
    o, _ = _lib()
    exe = os.path.join(tmp_path, "tuner_table")
    lib_dir = os.path.dirname(o.abi.LIB_PATH)
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "tuner_table.c"), "-L", lib_dir, "-lrcwa_b200",
                    "-Wl,-rpath," + lib_dir, "-o", exe], check=True)
    out = subprocess.run([exe, os.path.join(tmp_path, "table.txt")], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == "ok"
