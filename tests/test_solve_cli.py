"""Argument handling of the command-line solver (no GPU needed: these fail
before any device work)."""

import pytest

from scratch_wadge_b200 import solve


def test_mesh_file_needs_dimension(capsys):
    with pytest.raises(SystemExit) as e:
        solve.main(["--mesh-filename", "m.msh"])
    assert e.value.code == 2
    assert "--dim" in capsys.readouterr().err


def test_unknown_case_rejected():
    with pytest.raises(SystemExit):
        solve.main(["--case", "hexes"])


def test_cases_cover_the_workload_families():
    assert {c["ic"] for c in solve.CASES.values()} == {"vortex", "taylor_green", "density_wave"}
    assert solve.CASES["tg3d"]["n"] == 16 and solve.CASES["curved3d"]["curved"]
