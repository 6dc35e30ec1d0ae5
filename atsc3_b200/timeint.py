"""Time de-interleavers of A/322 fused into the GPU demapper's cell load.

The reference receiver de-interleaves a PLP's cells on the host before it
demaps them: the hybrid time interleaver's twisted block de-interleaver
(``lab/m6_tbi.py:75-88`` ``fec_block``, applied to a whole TI block as one
cached index gather in ``lab/m9_fast.py:1087-1093``) and the convolutional
time interleaver (``lab/m10_cti.py:126-141`` ``deinterleave``).  Here the
demapper reads each FEC Block cell straight from its position in the
received stream (``atsc3_demap_gather``, ``csrc/timeint.cu``): no
de-interleaved copy of the cells is written.

Index maps:

* twisted block interleaver (A/322 7.1.5.4), TI block of ``nrows`` rows
  (cells per FEC Block) by ``ncols`` columns (FEC Blocks, the first
  ``n_virtual`` of them virtual): output cell i reads memory position
  theta_i = nrows*C_i + R_i with R_i = i mod nrows, C_i = ((R_i mod ncols)
  + i div nrows) mod ncols, skipping theta_i < n_virtual*nrows;
* convolutional interleaver (A/322 7.1.4): pre-interleaver cell i leaves at
  q(i) = i + nrows*((start_row + i) mod nrows).
"""
from __future__ import annotations

import numpy as np

from . import demap as DM
from . import native as N


def _torch():
    import torch
    return torch


def tbi_read_order(nrows, ncols, n_virtual=0):
    """Memory index (data FEC Blocks only) of every transmitted cell of one TI
    block, in transmission order (A/322 7.1.5.4; lab/m6_tbi.py:46-58)."""
    i = np.arange(nrows * ncols, dtype=np.int64)
    r = i % nrows
    c = ((r % ncols) + i // nrows) % ncols
    theta = nrows * c + r
    keep = theta >= n_virtual * nrows
    return theta[keep] - n_virtual * nrows


def tbi_positions(nrows, ncols, n_virtual=0):
    """(ncols - n_virtual, nrows) transmitted position, inside the TI block,
    of cell r of data FEC Block j (the inverse of tbi_read_order)."""
    order = tbi_read_order(nrows, ncols, n_virtual)
    pos = np.empty(order.size, np.int64)
    pos[order] = np.arange(order.size)
    return pos.reshape(ncols - n_virtual, nrows)


class HybridTI:
    """Twisted block de-interleaving of ``nti`` consecutive TI blocks of a
    PLP: ``nrows`` cells per FEC Block, ``ncols`` FEC Blocks per TI block
    (``n_virtual`` of them virtual), TI block t starting at ``offset +
    t*per_ti`` in the received cell stream (``per_ti`` defaults to
    nrows*(ncols - n_virtual)).  FEC Block b = data Block b mod (ncols -
    n_virtual) of TI block b div (ncols - n_virtual)."""

    def __init__(self, nrows, ncols, nti=1, n_virtual=0, per_ti=None, offset=0):
        if not (0 <= n_virtual < ncols) or nrows < 1 or nti < 1:
            raise ValueError("need nrows >= 1, nti >= 1, 0 <= n_virtual < ncols")
        self.nrows, self.ncols, self.nti = int(nrows), int(ncols), int(nti)
        self.n_virtual, self.offset = int(n_virtual), int(offset)
        self.per_ti = int(per_ti if per_ti is not None
                          else nrows * (ncols - n_virtual))
        if self.per_ti < nrows * (ncols - n_virtual):
            raise ValueError("per_ti smaller than the TI block")
        self.nblk = self.nti * (self.ncols - self.n_virtual)
        self.ncell = self.nrows

    def index(self):
        """(nblk, nrows) int32 source positions in the received stream."""
        pos = tbi_positions(self.nrows, self.ncols, self.n_virtual)
        t = np.arange(self.nti, dtype=np.int64)[:, None, None]
        idx = self.offset + t * self.per_ti + pos[None]
        return idx.reshape(self.nblk, self.nrows).astype(np.int32)

    def launch_args(self):
        """(gather_mode, p0, p1, p2) of atsc3_demap_gather: the closed form
        without virtual Blocks, else an index table."""
        if self.n_virtual == 0:
            return 1, self.offset, self.ncols, self.per_ti
        return 0, 0, 0, 0

    def stream_cells(self):
        return self.offset + self.nti * self.per_ti

    def interleave(self, blocks):
        """Transmit side (tests and synthetic streams): (nblk, nrows) FEC
        Block cells -> the received stream (torch or numpy 1-D)."""
        torch = _torch()
        idx = torch.as_tensor(self.index().ravel().astype(np.int64),
                              device=blocks.device)
        out = torch.zeros(self.stream_cells(), dtype=blocks.dtype,
                          device=blocks.device)
        out[idx] = blocks.reshape(-1)
        return out


class ConvolutionalTI:
    """Convolutional de-interleaving: ``nrows`` delay lines, commutator at
    ``start_row`` for the first received cell, FEC Block 0 starting at
    pre-interleaver cell ``C`` (A/322 9.3.9.1; lab/m10_cti.py:144-151)."""

    def __init__(self, nrows, start_row, C=0, nblk=1, ncell=1):
        if nrows < 1 or start_row < 0 or C < 0:
            raise ValueError("need nrows >= 1, start_row >= 0, C >= 0")
        self.nrows, self.start_row, self.C = int(nrows), int(start_row), int(C)
        self.nblk, self.ncell = int(nblk), int(ncell)

    def source(self, i):
        i = np.asarray(i, np.int64)
        return i + self.nrows * ((self.start_row + i) % self.nrows)

    def index(self, ncells):
        """(nblk, ncell) int32 source positions, -1 past the stream."""
        i = self.C + np.arange(self.nblk * self.ncell, dtype=np.int64)
        q = self.source(i)
        q[q >= ncells] = -1
        return q.reshape(self.nblk, self.ncell).astype(np.int32)

    def launch_args(self):
        return 2, self.C, self.nrows, self.start_row

    def interleave(self, pre, ncells):
        """Transmit side: pre-interleaver cells (1-D, from cell 0) -> the
        received stream of ``ncells`` cells (positions fed from before cell
        0 stay 0)."""
        torch = _torch()
        q = torch.arange(ncells, device=pre.device, dtype=torch.int64)
        i = q - self.nrows * ((self.start_row + q) % self.nrows)
        ok = (i >= 0) & (i < pre.numel())
        out = torch.zeros(ncells, dtype=pre.dtype, device=pre.device)
        out[ok] = pre[i[ok]]
        return out


def demap_deinterleave(stream, ti, mod, rate, n, sigma2=None, out=None,
                       stream_id=None, table=False):
    """De-interleave + demap: ``stream`` is the received PLP cell stream
    (1-D complex64 CUDA tensor), ``ti`` a HybridTI or ConvolutionalTI;
    ``sigma2``: float, a 1-D tensor per received cell, or (nblk,) per FEC
    Block.  Returns (nblk, n) float32 LLRs in codeword order.  ``table``
    forces the index-table mode (tests)."""
    torch = _torch()
    from . import codes as C
    if stream.dtype != torch.complex64 or stream.device.type != "cuda" or \
            stream.dim() != 1 or not stream.is_contiguous():
        raise TypeError("stream must be a contiguous 1-D CUDA complex64 tensor")
    stream = stream.resolve_conj()
    nb = C.MOD_BITS[mod]
    nblk, ncell = ti.nblk, ti.ncell
    if ncell != C.cells_per_block(n, mod):
        raise ValueError("TI rows must equal the cells of one FEC Block")
    dev = stream.device
    if out is None:
        out = torch.empty((nblk, n), dtype=torch.float32, device=dev)
    mode, p0, p1, p2 = ti.launch_args()
    src = None
    if table or mode == 0:
        idx = ti.index() if isinstance(ti, HybridTI) else ti.index(stream.numel())
        src = torch.from_numpy(idx).to(dev)
        mode, p0, p1, p2 = 0, 0, 0, 0
    s2mode, s2t, s2s = 0, None, 1.0
    if isinstance(sigma2, (int, float)):
        s2s = float(sigma2)
    elif sigma2 is not None:
        s2t = sigma2.to(dev, torch.float32).contiguous()
        if s2t.numel() == stream.numel():
            s2mode = 1
        elif s2t.numel() == nblk:
            s2mode = 2
        else:
            raise ValueError("sigma2 must be a scalar, per received cell or per block")
    else:
        raise ValueError("sigma2 is required (no estimate across a TI block)")
    st = stream_id if stream_id is not None else torch.cuda.current_stream(dev).cuda_stream
    N.call("atsc3_demap_gather", torch.view_as_real(stream).data_ptr(),
           stream.numel(), nblk, ncell,
           DM.device_points(mod, rate, dev).data_ptr(), nb, mode, N.ptr(src),
           p0, p1, p2, s2mode, N.ptr(s2t), s2s,
           DM.device_lam_of_q(n, mod, rate, dev).data_ptr(),
           out.data_ptr(), out.stride(0), st)
    if src is not None:
        out._ti_src = src          # keep the table alive until the launch ran
    return out
