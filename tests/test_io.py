"""The .sd2 / .af2 readers and writers: round trips, and byte-for-byte agreement with files written by the
reference's own DensityFunction::WriteToDisk / OrdinateFlux::WriteToDisk (compiled reference)."""
import os

import numpy as np
import pytest

from conftest import to_oracle
from idcsweep import io
from idcsweep.problems import random_problem


def test_round_trip(tmp_path):
    P = random_problem(7, 5, 2, 8, seed=1)
    phi = np.random.default_rng(0).standard_normal(P.phi_shape())
    io.write_sd2(str(tmp_path / "a.sd2"), phi, P.ax, P.bx, P.ay, P.by)
    h, got = io.read_sd2(str(tmp_path / "a.sd2"))
    assert (h.nx, h.ny, h.dg_degree) == (7, 5, 2) and (h.ax, h.bx, h.ay, h.by) == (P.ax, P.bx, P.ay, P.by)
    assert np.array_equal(got, phi)
    io.write_af2(str(tmp_path / "a.af2"), P.source, P.ax, P.bx, P.ay, P.by, "level-symmetric", 8)
    h, got = io.read_af2(str(tmp_path / "a.af2"))
    assert h.ordinate_type == "level-symmetric" and h.ang_order == 8 and got.shape == P.source.shape
    assert np.array_equal(got, P.source)


def test_reader_rejects_garbage(tmp_path):
    p = tmp_path / "bad.sd2"
    p.write_bytes(b"\x01\x02\x03")
    with pytest.raises(OSError):
        io.read_sd2(str(p))


def test_files_of_the_reference(reference, tmp_path):
    P = random_problem(6, 4, 1, 4, seed=3)
    phi = np.random.default_rng(2).standard_normal(P.phi_shape())
    with reference.open(to_oracle(P), P.dt) as h:
        h.write_sd(phi, str(tmp_path / "ref.sd2"))
        h.write_af(P.source, str(tmp_path / "ref.af2"))
    hd, got = io.read_sd2(str(tmp_path / "ref.sd2"))
    assert (hd.nx, hd.ny, hd.dg_degree) == (P.nx, P.ny, P.p)
    assert np.array_equal(got, phi)
    io.write_sd2(str(tmp_path / "ours.sd2"), phi, P.ax, P.bx, P.ay, P.by)
    assert (tmp_path / "ours.sd2").read_bytes() == (tmp_path / "ref.sd2").read_bytes()
    ha, gpsi = io.read_af2(str(tmp_path / "ref.af2"))
    assert np.array_equal(gpsi, P.source)
    io.write_af2(str(tmp_path / "ours.af2"), P.source, P.ax, P.bx, P.ay, P.by, ha.ordinate_type, ha.ang_order)
    assert (tmp_path / "ours.af2").read_bytes() == (tmp_path / "ref.af2").read_bytes()
