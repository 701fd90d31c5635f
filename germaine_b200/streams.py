"""A frequency batch split over several engines of one GPU, each with its own
CUDA stream, driven from host threads (the C-ABI calls release the
interpreter lock).  One engine runs every tree level of the whole batch as
one launch per kernel; the upper levels hold few fronts (1 .. 16 per
frequency at 841 x 227) and leave most of the 148 SMs idle while their
dependent launches run one after another.  Two engines with half the
frequencies each run those latency-bound stretches side by side, while the
wide lower levels of one fill the SMs the other leaves free.

Same kernels and results as one engine; the outputs are stitched back in
frequency order.
"""
from __future__ import annotations

from concurrent.futures import ThreadPoolExecutor

import numpy as np

from .engine import Engine


def split_frequencies(nf: int, parts: int):
    """Contiguous blocks of the frequency index range, as even as possible."""
    parts = max(1, min(parts, nf))
    base, extra = divmod(nf, parts)
    out, start = [], 0
    for p in range(parts):
        size = base + (1 if p < extra else 0)
        out.append(range(start, start + size))
        start += size
    return out


class StreamedEngines:
    """`parts` engines over one grid (same configuration), frequencies split
    in contiguous blocks; factor + forward run concurrently."""

    def __init__(self, nx, ny, dh, npml, parts: int = 2, **kw):
        self.engines = [Engine(nx, ny, dh, npml, **kw) for _ in range(parts)]
        self.pool = ThreadPoolExecutor(max_workers=parts)
        self.blocks = None

    def close(self):
        for e in self.engines:
            e.close()
        self.pool.shutdown()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_model(self, mat0, mat1):
        for e in self.engines:
            e.set_model(mat0, mat1)

    def factor(self, freqs):
        f = np.asarray(freqs, np.float32)
        self.blocks = split_frequencies(f.size, len(self.engines))
        list(self.pool.map(lambda i: self.engines[i].factor(f[list(self.blocks[i])]), range(len(self.blocks))))

    def forward(self, src_x, src_y, rec_x, rec_y, seis_out=None):
        """Seismograms [nf][nshots][ntr] complex64 of all frequencies (or into
        seis_out, a host or device array of that shape)."""
        def one(i):
            b = self.blocks[i]
            view = seis_out[b.start:b.stop] if seis_out is not None else None   # frequency-outer: contiguous
            s, _ = self.engines[i].forward(src_x, src_y, rec_x, rec_y, seis_out=view)
            return s
        parts = list(self.pool.map(one, range(len(self.blocks))))
        return seis_out if seis_out is not None else np.concatenate(parts, axis=0)

    def stats(self):
        return [e.stats() for e in self.engines]

    def refine_report(self):
        out = []
        for e in self.engines:
            out.extend(e.refine_report())
        return out
