"""The static autotuner's cache file (host only): tc_autotune_load reads version-3 lines
("log2n log2m log2maxdplus warp_max lane_max chunk blocks_per_sm packed_max") and version-2 lines
without packed_max (which then get no packed walks), tc_autotune_lookup returns the entry of a
graph's bucket (log2 n, log2 m, log2 max out-degree), and tc_autotune_save writes back what was
loaded."""
import ctypes

from custingeralg_b200 import native as N


def lookup(n, m, maxd):
    s = N.Sched()
    st = N.lib().tc_autotune_lookup(n, m, maxd, ctypes.byref(s))
    return st, s


def test_load_lookup_save_roundtrip(tmp_path):
    p = tmp_path / "tune.txt"
    p.write_text("# tc autotune v3: log2n log2m log2maxdplus warp_max lane_max chunk blocks_per_sm packed_max\n"
                 "20 24 9 128 4 32 6 64\n"
                 "# a version-2 line\n"
                 "16 20 5 32 16 128 0\n")
    assert N.lib().tc_autotune_load(str(p).encode()) == N.TC_OK
    st, s = lookup(1 << 20, 1 << 24, 1 << 9)
    assert st == N.TC_OK
    assert (s.warp_max_deg, s.lane_max_deg, s.chunk, s.blocks_per_sm, s.packed_max_deg) == (128, 4, 32, 6, 64)
    st, s = lookup((1 << 16) + 5, (1 << 20) + 7, 40)   # same bucket: floor(log2) of each figure
    assert st == N.TC_OK
    assert (s.warp_max_deg, s.lane_max_deg, s.chunk, s.blocks_per_sm, s.packed_max_deg) == (32, 16, 128, 0, 0)
    # a bucket with no entry: the default scheduler and a state error
    st, s = lookup(1 << 10, 1 << 12, 4)
    assert st == N.TC_ERR_STATE
    d = N.default_sched()
    assert (s.warp_max_deg, s.lane_max_deg, s.packed_max_deg) == (d.warp_max_deg, d.lane_max_deg, d.packed_max_deg)
    q = tmp_path / "saved.txt"
    assert N.lib().tc_autotune_save(str(q).encode()) == N.TC_OK
    lines = [ln.split() for ln in q.read_text().splitlines() if not ln.startswith("#")]
    assert ["20", "24", "9", "128", "4", "32", "6", "64"] in lines
    assert ["16", "20", "5", "32", "16", "128", "0", "0"] in lines


def test_load_errors(tmp_path):
    assert N.lib().tc_autotune_load(str(tmp_path / "missing.txt").encode()) == N.TC_ERR_INVALID_ARG
    p = tmp_path / "empty.txt"
    p.write_text("# nothing\nnot numbers\n")
    assert N.lib().tc_autotune_load(str(p).encode()) == N.TC_ERR_INVALID_ARG
