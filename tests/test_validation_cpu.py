"""LDBC validation-file helpers (graphhet_b200.validation) on the CPU: the
writer's format and the checker's rules (checker.hpp)."""
from graphhet_b200 import validation as V


def test_write_read_and_check(tmp_path):
    names = ["a", "b", "c", "d"]
    p = str(tmp_path / "x.bfs")
    V.write(p, "bfs", names, [0, 1, 2**31 - 1, 2])
    assert V.read(p)[2] == ("c", "9223372036854775807")
    assert V.check(p, "bfs", names, [0, 1, 2**31 - 1, 2])[0]
    assert not V.check(p, "bfs", names, [0, 1, 2, 2])[0]
    p = str(tmp_path / "x.sssp")
    V.write(p, "sssp", names, [0.0, 0.5, V.DBL_MAX, 1.25])
    assert V.read(p)[2] == ("c", "infinity")
    assert V.check(p, "sssp", names, [0.0, 0.50001, V.DBL_MAX, 1.25])[0]
    assert not V.check(p, "sssp", names, [0.0, 0.6, V.DBL_MAX, 1.25])[0]
    p = str(tmp_path / "x.wcc")
    V.write(p, "wcc", names, [0, 0, 2, 2])
    assert V.check(p, "wcc", names, [1, 1, 3, 3])[0]      # same partition, other labels
    assert not V.check(p, "wcc", names, [0, 1, 2, 2])[0]
