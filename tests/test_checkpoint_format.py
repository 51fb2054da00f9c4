"""The Python reader of the checkpoint format against a file built here from
the documented layout (no GPU): header fields, array placement, checksum."""
import numpy as np
import pytest

from hydrocode_astro1_b200.checkpoint import HEADER, fnv1a64, read_checkpoint


def write(path, shape, precision, gravity, corrupt=False):
    n = int(np.prod(shape))
    word = np.float64 if precision == 0 else np.float32
    rng = np.random.default_rng(5)
    state = rng.standard_normal((5,) + shape).astype(word)
    parts = [state.tobytes()]
    phi = phig = None
    if gravity:
        phi = rng.standard_normal(shape)
        phig = rng.standard_normal(shape)
        parts += [phi.tobytes(), phig.tobytes()]
    payload = b"".join(parts)
    h = np.zeros((), dtype=HEADER)
    h["magic"], h["version"], h["header_bytes"] = b"HCCKPT01", 1, HEADER.itemsize
    h["nx"], h["ny"], h["nz"] = shape
    h["precision"], h["gravity"], h["parity"], h["step"], h["t"] = precision, gravity, 1, 7, 0.25
    h["lo"], h["hi"], h["gamma"], h["G"] = (0, 0, 0), (1, 1, 1), 5 / 3, 1.0
    h["payload_bytes"], h["checksum"] = len(payload), fnv1a64(payload) ^ (1 if corrupt else 0)
    with open(path, "wb") as f:
        f.write(h.tobytes() + payload)
    assert n * 5 * np.dtype(word).itemsize + (16 * n if gravity else 0) == len(payload)
    return state, phi, phig


@pytest.mark.parametrize("precision,gravity", [(0, 1), (1, 1), (1, 0)])
def test_reader_layout(tmp_path, precision, gravity):
    p = str(tmp_path / "x.ckpt")
    state, phi, phig = write(p, (3, 4, 5), precision, gravity)
    ck = read_checkpoint(p, verify=True)
    assert ck["shape"] == (3, 4, 5) and int(ck["step"]) == 7 and float(ck["t"]) == 0.25
    assert np.array_equal(ck["state"], state)
    if gravity:
        assert np.array_equal(ck["phi"], phi) and np.array_equal(ck["phig"], phig)
    else:
        assert "phi" not in ck


def test_reader_checksum(tmp_path):
    p = str(tmp_path / "y.ckpt")
    write(p, (3, 4, 5), 0, 1, corrupt=True)
    with pytest.raises(ValueError, match="checksum"):
        read_checkpoint(p, verify=True)


def test_fnv_known_answer():
    # FNV-1a 64 published test values
    assert fnv1a64(b"") == 0xcbf29ce484222325
    assert fnv1a64(b"a") == 0xaf63dc4c8601ec8c
    assert fnv1a64(b"foobar") == 0x85944171f73967e8
