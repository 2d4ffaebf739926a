"""SDF snapshots and checkpoints (nlnhost.h nln_sdf_*): the reference's
outbody records and header layout, written and read back.  CPU only."""
import numpy as np
import pytest


def test_round_trip_with_and_without_accelerations(tmp_path):
    from pgrav import sdf
    rng = np.random.default_rng(1)
    n = 70000   # more than one write buffer
    pos = rng.normal(size=(n, 3)).astype(np.float32)
    vel = rng.normal(size=(n, 3)).astype(np.float32)
    m = rng.uniform(0.5, 1.5, n).astype(np.float32)
    ident = rng.permutation(n).astype(np.int64) * 3 + 7
    acc = rng.normal(size=(n, 4)).astype(np.float32)
    hdr = {"npart": (sdf.INT64, n), "iter": (sdf.INT, 12), "tpos": (sdf.DOUBLE, 0.123456789012345),
           "L0": (sdf.FLOAT, 1.0), "custom": 5}
    for a in (None, acc):
        p = tmp_path / ("acc.sdf" if a is not None else "plain.sdf")
        sdf.write(p, pos, vel, m, ident=ident, acc_phi=a, header=hdr)
        h, b = sdf.read(p)
        assert h["npart"] == n and h["iter"] == 12 and h["custom"] == 5
        assert h["tpos"] == 0.123456789012345 and h["L0"] == 1.0
        assert np.array_equal(b["pos"], pos) and np.array_equal(b["vel"], vel)
        assert np.array_equal(b["mass"], m) and np.array_equal(b["ident"], ident)
        assert ("acc_phi" in b) == (a is not None)
        if a is not None:
            assert np.array_equal(b["acc_phi"], acc)
        # the record size is the packed outbody's: 36 or 52 bytes
        text = open(p, "rb").read()
        data = text[text.index(b"# SDF-EOH\n") + len(b"# SDF-EOH\n"):]
        assert len(data) == n * (52 if a is not None else 36)


def test_header_is_the_reference_layout(tmp_path):
    from pgrav import sdf
    p = tmp_path / "h.sdf"
    sdf.write(p, np.zeros((2, 3)), np.zeros((2, 3)), 1.0, header={"iter": (sdf.INT, 1)})
    head = open(p, "rb").read().split(b"# SDF-EOH")[0].decode()
    assert head.startswith("# SDF 1.0\nparameter byteorder = 0x78563412;\nint iter = 1;\n")
    for field in ("float mass;", "float x, y, z;", "float vx, vy, vz;", "int64_t ident;", "}[2];"):
        assert field in head
    assert "#\f\n" in head


def test_malformed_files_are_refused(tmp_path):
    from pgrav import sdf
    p = tmp_path / "bad.sdf"
    p.write_bytes(b"# SDF 1.0\nint n = 3;\n")          # no end of header
    with pytest.raises(IOError, match="end-of-header"):
        sdf.read(p)
    p.write_bytes(b"# SDF 1.0\nstruct {\n double x;\n}[3];\n#\f\n# SDF-EOH\n")
    with pytest.raises(IOError, match="unsupported"):
        sdf.read(p)
    good = tmp_path / "good.sdf"
    sdf.write(good, np.zeros((10, 3)), np.zeros((10, 3)), 1.0)
    raw = open(good, "rb").read()
    p.write_bytes(raw[:-5])                               # truncated records
    with pytest.raises(IOError, match="ends before"):
        sdf.read(p)
