"""External source wavelet (READ_WAVELET = 1): the host drop-in for
read_stf_dft (src/read_stf_dft.c:12-73) against the reference's own compiled
function, bit for bit, on SU traces written here (no GPU needed)."""
import numpy as np
import pytest

import oracle as O
from germaine_b200 import engine as E

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")


def write_su(path, samples, dt_units):
    """One SU trace: a 240-byte header with ns (bytes 114-115) and dt
    (bytes 116-117) as native unsigned shorts, then the float samples."""
    hdr = bytearray(240)
    hdr[114:116] = np.array([len(samples)], np.uint16).tobytes()
    hdr[116:118] = np.array([dt_units], np.uint16).tobytes()
    with open(path, "wb") as f:
        f.write(bytes(hdr))
        f.write(np.asarray(samples, np.float32).tobytes())


def ricker(ns, dt, fc, t0):
    t = np.arange(ns) * dt - t0
    a = (np.pi * fc * t) ** 2
    return ((1 - 2 * a) * np.exp(-a)).astype(np.float32)


@pytest.mark.parametrize("physics,dt_units,freqs,fc", [
    (1, 1000, [2.0, 3.0, 7.5, 11.0], 8.0),        # acoustic: dt in microseconds (1 ms)
    (2, 500, [4.0, 13.0], 15.0),                  # SH
    (4, 100, [1.0e8, 2.2e8, 4.0e8], 2.0e8),       # TE: dt in nanoseconds (0.1 ns)
])
def test_stf_dft_matches_reference(tmp_path, physics, dt_units, freqs, fc):
    dt = dt_units / (1e6 if physics <= 3 else 1e12)
    rng = np.random.default_rng(physics)
    for trial, ns in enumerate((1, 2, 257, 1500)):
        s = ricker(ns, dt, fc, 1.2 / fc) + rng.normal(0, 1e-3, ns).astype(np.float32)
        p = tmp_path / f"w{trial}.su"
        write_su(p, s, dt_units)
        for f in freqs:
            ours = E.stf_dft(str(p), physics, f)
            ref = O.ref_stf_dft(str(p), physics, f)
            assert np.complex64(ours) == np.complex64(ref), (ns, f, ours, ref)


def test_stf_dft_errors(tmp_path):
    from germaine_b200 import GmError
    with pytest.raises(GmError):
        E.stf_dft(str(tmp_path / "missing.su"), 1, 5.0)
    short = tmp_path / "short.su"
    short.write_bytes(b"\0" * 100)
    with pytest.raises(GmError):
        E.stf_dft(str(short), 1, 5.0)
