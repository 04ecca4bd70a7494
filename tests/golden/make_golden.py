"""Generate the FFTPACK golden vectors in tests/golden/fftpack_rfft.npz.

scipy.fftpack.rfft/irfft wrap FFTPACK, the same library the reference ships
as src/fftpack.f (RFFTF/RFFTB, packed half-complex order).  Run once; the
.npz is committed so the tests do not need scipy at run time.
"""
import os

import numpy as np
import scipy.fftpack as sf

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    rng = np.random.RandomState(20240611)
    out = {}
    for n in (2, 4, 8, 16, 32, 64, 256, 6, 12, 30, 384):
        x = rng.randn(n)
        out[f"x{n}"] = x
        out[f"f{n}"] = sf.rfft(x)                 # RFFTF
        out[f"b{n}"] = sf.irfft(sf.rfft(x)) * n   # RFFTB o RFFTF = n * identity
        r = rng.randn(n)
        out[f"r{n}"] = r
        out[f"rb{n}"] = sf.irfft(r) * n           # RFFTB of an arbitrary packed vector
    np.savez_compressed(os.path.join(HERE, "fftpack_rfft.npz"), **out)


if __name__ == "__main__":
    main()
