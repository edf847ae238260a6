"""The checked build (lib/libs615_checked.so) on the device (GPU).

Its kernels compare every table cell, work item, unit, shard and key index
with its bound and record a failed check in a flag word instead of making the
access.  This runs the main paths through that build -- class-5 units and
plants against an oracle-built table, the one-launch-per-unit form, a mixed
queue of class 2-5 units, job rows and (6,1,7) candidates, the device xor
builder (binned incidence, list peel) and a shard set -- and requires no flag
set and the results of the default build (the oracle's for the class-5 batch).  The checked build is loaded in a
child process (the library is chosen when s615 is imported): this file run as
a script with S615_CHECKED=1.
"""
import json
import os
import subprocess
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def test_default_build_is_not_checked():
    import s615
    assert s615.lib().s615_checked_build() == 0


@pytest.mark.gpu
def test_checked_build_sets_no_flag(tmp_path):
    env = dict(os.environ, S615_CHECKED="1")
    p = subprocess.run([sys.executable, os.path.abspath(__file__), str(tmp_path)], env=env,
                       capture_output=True, text=True, timeout=1200)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-4000:]
    res = json.loads(p.stdout.strip().splitlines()[-1])
    assert res["checked_build"] == 1
    assert res["flags"] == {k: 0 for k in res["flags"]}, res
    assert res["cls5_equal_oracle"] and res["plain_equal"] and res["mixed_equal_parts"]
    assert res["build_fn0"]


def _child(tmp):
    sys.path[:0] = [os.path.join(ROOT, "six-one-five_b200"), os.path.join(ROOT, "oracle"), HERE]
    import numpy as np

    import orc
    import s615
    import workloads as W
    from test_gpu_cls5 import oracle_units, sorted_hits

    lib = s615.lib()
    out = {"checked_build": int(lib.s615_checked_build()), "flags": {}}
    with s615.Engine(0) as eng:
        # class-5 units and plants on an oracle-built table: the oracle's hits
        N = 715
        t = orc.Table.build_pairs(N, 16)
        path = os.path.join(tmp, "orc.bin")
        t.save(path)
        tid = eng.load_table(path, N)
        units = W.cls5_units(1000, 30000)
        plants = W.plants(8, 0, 1000, 30000, N)
        arr, n = W.unit_array(units, plants, N)
        hits, ctr = eng.cls5_run(tid, arr, n)
        oarr, on = oracle_units(units, plants, N)
        ohits, (calls, gated, probes) = orc.cls5_run(t, oarr, on)
        out["cls5_equal_oracle"] = bool((ctr.calls, ctr.gated, ctr.probes) == (calls, gated, probes)
                                        and np.array_equal(sorted_hits(hits), sorted_hits(ohits)))
        out["flags"]["cls5"] = eng.check_flags()
        # the plain form (one launch per unit) on the first 40 units: the batched results
        ph, pc = eng.cls5_run(tid, arr, 40, flags=s615.F_PLAIN)
        dh, dc = eng.cls5_run(tid, arr, 40)
        out["plain_equal"] = bool(np.array_equal(sorted_hits(ph), sorted_hits(dh))
                                  and (pc.calls, pc.probes) == (dc.calls, dc.probes) and dc.probes > 0)
        out["flags"]["plain"] = eng.check_flags()

        # one queue of class 2-5 units, job rows and (6,1,7) candidates == the parts alone
        Nm = 26000 // 42 + 1
        tm = eng.build_table(Nm, 16)
        mixed = W.mixed_units(400, 9, 24001, 26000)
        ma, mn = W.mixed_unit_array(mixed, [], [], Nm)
        jobs, jn, _ = s615.expand_units([(c, B, u) for c, B, u in mixed[:40] if c in (2, 3, 4)])
        c7, n7 = s615.candidates617(24329)
        allu = (s615.Unit * (mn + jn + n7))()
        for i in range(mn):
            allu[i] = ma[i]
        for i in range(jn):
            allu[mn + i] = jobs[i]
        for i in range(n7):
            allu[mn + jn + i] = c7[i]
        hm, cm = eng.run(tm, allu, mn + jn + n7)
        parts = 0
        for lo, k in ((0, mn), (mn, jn), (mn + jn, n7)):
            sub = (s615.Unit * max(k, 1))(*[allu[lo + i] for i in range(k)])
            _, c = eng.run(tm, sub, k)
            parts += c.probes
        out["mixed_equal_parts"] = bool(cm.probes == parts and cm.probes > 0)
        out["flags"]["mixed"] = eng.check_flags()
        eng.free_table(tm)

        # the device builder (list peel), a shard set, and the queries on both: no false negative
        keys = np.unique(np.array([(i**6 + j**6) % 2**64 for i in range(1, 301) for j in range(i, 301)],
                                  dtype=np.uint64))
        tb = eng.build_table(300, 16)
        ok = bool(eng.query(tb, keys).all())
        eng.free_table(tb)
        out["flags"]["build"] = eng.check_flags()
        ts = eng.build_table_sharded(300, 16, 3)
        ok = ok and bool(eng.query(ts, keys).all())
        eng.free_table(ts)
        out["flags"]["shards"] = eng.check_flags()
        out["build_fn0"] = ok
        eng.free_table(tid)
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    _child(sys.argv[1])
