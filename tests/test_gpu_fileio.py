"""Snapshot output in the reference's format (fileio_MPI_IO.c:63-118):
output/sim-N.bin = x, y, z interleaved as doubles in original particle order,
checked bit for bit against the positions read back through the C ABI; and
the asynchronous read-back of the output frame."""
import os

import numpy as np
import pytest

from sphpc_b200 import Simulation

pytestmark = pytest.mark.gpu


def test_snapshots_match_positions(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    with Simulation("small_obstacle") as sim:
        f = sim.fileio_open()
        assert f.file_num == 0 and os.path.isdir(tmp_path / "output")
        expect = []
        for k in range(3):
            st = sim.fetch(["x", "y", "z"])
            expect.append(np.stack([st["x"], st["y"], st["z"]], axis=1).ravel())
            sim.write_particles(f)       # returns before the file is on disk
            sim.step(2)                  # the snapshot is of the state at the call
        sim.fileio_wait(f)
        assert f.file_num == 3
        sim.fileio_close(f)
    for k in range(3):
        got = np.fromfile(tmp_path / "output" / f"sim-{k}.bin", dtype=np.float64)
        assert got.shape == expect[k].shape
        assert np.array_equal(got, expect[k])
    assert not np.array_equal(expect[0], expect[2])


def test_async_read_back_is_the_state_it_was_taken_from():
    """sphpc_update_host_fields_async: the host arrays receive the state of
    the moment of the call even when steps follow before host_wait, and a
    read-back after those steps equals the synchronous one."""
    fields = ["x", "y", "z", "density"]
    with Simulation("small_dam") as sim:
        sim.step(3)
        sim.fetch_fields(fields)
        want = {f: sim.host(f).copy() for f in fields}
        for f in fields:
            sim.host(f)[:] = 0.0
        sim.fetch_fields_async(fields)
        sim.step(2)
        sim.host_wait()
        for f in fields:
            np.testing.assert_array_equal(sim.host(f), want[f], err_msg=f)
        sim.fetch_fields_async(fields)
        sim.host_wait()
        later = {f: sim.host(f).copy() for f in fields}
        assert not np.array_equal(later["y"], want["y"])
        sim.fetch_fields(fields)
        for f in fields:
            np.testing.assert_array_equal(sim.host(f), later[f], err_msg=f)
        assert sim.device_errors() == 0
