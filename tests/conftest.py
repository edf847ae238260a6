import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "six-one-five_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden", "golden.json")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run on the B200 box)")


@pytest.fixture(scope="session")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def engine():
    import s615
    eng = s615.Engine(0)
    yield eng
    eng.close()


@pytest.fixture(scope="session")
def table_dir(tmp_path_factory):
    return tmp_path_factory.mktemp("tables")


@pytest.fixture(scope="session")
def oracle_table(table_dir):
    """Oracle-built pair tables (byte-identical to the reference builder),
    saved to files and cached per (N, r)."""
    import orc
    cache = {}

    def get(N, r):
        key = (N, r)
        if key not in cache:
            t = orc.Table.build_pairs(N, r)
            path = str(table_dir / f"orc_N{N}_r{r}.bin")
            t.save(path)
            cache[key] = (t, path)
        return cache[key]

    return get
