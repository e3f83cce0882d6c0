"""Exact multiprecision products through a residue number system, on B200 tensor cores.

Drop-in for ``sdpvibe.rns`` (sdpvibe/rns.py): the same moduli, residue format (int8 hi/lo planes,
r = 128 hi + lo centred) and int16 accumulator, computed by libsdpv_b200:

* ``RNS.residues``   -> sdpv_residues  (tcgen05 byte-by-table product, one HBM pass)
* ``RNS.accumulate`` -> sdpv_rns_gemm  (TMA + tcgen05 int8 GEMM, modular reduction in the epilogue)
* ``RNS.crt_block``  -> sdpv_crt_block (pre-pass, tcgen05 digit product and carry in one kernel)
"""
import ctypes

import torch

from . import _lib

dev = "cuda"


class RNS:
    """Moduli and device tables for products of L-limb integers with inner dimension <= 2^17
    (sdpvibe/rns.py:163-191).  G: the moduli count is the least multiple of G primes that meets the bound
    (the reference's G = 16 by default; 1, 2, 4 and 8 give fewer moduli and the same exact products)."""

    KPAD = 16

    def __init__(self, L, kmax=1 << 17, G=16):
        if kmax != 1 << 17 or G not in (1, 2, 4, 8, 16):
            raise ValueError("libsdpv_b200 contexts use kmax = 2^17 and groups of 1, 2, 4, 8 or 16 moduli")
        h = ctypes.c_void_p()
        _lib.call("sdpv_ctx_create_g", int(L), int(G), ctypes.byref(h))
        self._h = h
        n, E, W = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _lib.call("sdpv_ctx_query", h, ctypes.byref(n), ctypes.byref(E), ctypes.byref(W))
        self.L, self.G, self.NB = L, G, 4 * L
        self.n, self.E, self.W = n.value, E.value, W.value
        arr = (ctypes.c_int32 * self.n)()
        _lib.call("sdpv_ctx_moduli", h, ctypes.cast(arr, ctypes.c_void_p))
        self.mods = list(arr)
        M = 1
        for m in self.mods:
            M *= m
        self.M = M
        self.device = torch.cuda.current_device()
        self.m32 = torch.tensor(self.mods, dtype=torch.int32, device=dev)

    @property
    def handle(self):
        return self._h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib._lib is not None:
            try:
                _lib.lib().sdpv_ctx_destroy(h)
            except Exception:
                pass

    # ---- step 1: residues (sdpvibe/rns.py:196-214)
    def residues(self, X, k0, kc, g0=0, G=None, spread=False, unsigned=False):
        """X: (L, rows, K) int32 limb planes -> (Rhi, Rlo) (G, rows, kp) int8, kp = kc rounded up to 16.
        spread=True places the modulus planes an odd multiple of 2 KB apart (a strided view) so the
        2G output streams spread over the HBM channels; accumulate() accepts either layout.
        unsigned=True gives the GEMM's internal digits instead of the API's: the canonical residue
        r in [0, m) as hi = r >> 7, lo = r & 127 (uint8 planes); pass unsigned=True to accumulate too."""
        L, rows, K = X.shape
        assert L == self.L
        G = G or self.n
        kp = -(-kc // self.KPAD) * self.KPAD
        X = X.contiguous()
        dt = torch.uint8 if unsigned else torch.int8
        if spread:
            ps = plane_stride(rows * kp)
            buf_h = torch.empty((G * ps,), dtype=dt, device=X.device)
            buf_l = torch.empty_like(buf_h)
            Rhi = buf_h.as_strided((G, rows, kp), (ps, kp, 1))
            Rlo = buf_l.as_strided((G, rows, kp), (ps, kp, 1))
        else:
            ps = 0
            Rhi = torch.empty((G, rows, kp), dtype=dt, device=X.device)
            Rlo = torch.empty_like(Rhi)
        _lib.call("sdpv_residues_u8" if unsigned else "sdpv_residues", self._h, _lib.ptr(X), rows, K, k0, kc, g0, G,
                  _lib.ptr_strided(Rhi), _lib.ptr_strided(Rlo), ps, _lib.stream())
        return Rhi, Rlo

    def residues_rows(self, Xr, nI, Rp, k0, kc, g0=0, G=None):
        """residues(..., spread=True, unsigned=True) of operand rows (mpf.aligned_rows): entry (i, k) is row
        i * Rp + k0 + k of Xr; k0 a multiple of 128, g0 of 128; rows k0 + kc .. k0 + kp - 1 must be zero rows."""
        G = G or self.n
        kp = -(-kc // self.KPAD) * self.KPAD
        ps = plane_stride(nI * kp)
        buf_h = torch.empty((G * ps,), dtype=torch.uint8, device=Xr.device)
        buf_l = torch.empty_like(buf_h)
        Rhi = buf_h.as_strided((G, nI, kp), (ps, kp, 1))
        Rlo = buf_l.as_strided((G, nI, kp), (ps, kp, 1))
        _lib.call("sdpv_residues_rows", self._h, _lib.ptr(Xr), nI, Rp, k0, kc, g0, G, _lib.ptr_strided(Rhi),
                  _lib.ptr_strided(Rlo), ps, _lib.stream())
        return Rhi, Rlo

    # ---- step 2: accumulate residues of A @ Bt^T (sdpvibe/rns.py:217-224)
    def accumulate(self, Ahi, Alo, Bhi, Blo, acc, g0=0, nb=1, syrk=False, fresh=False, unsigned=False):
        """acc[g0:g0+G] += residues of A @ B^T; with nb > 1 the operands hold nb blocks stacked along rows.
        acc may have padded rows (acc.shape[2] >= N): its row stride is passed to the kernel.  fresh: the
        updated entries are overwritten (acc's content there is taken as zero and not read)."""
        G, Mt, KC = Ahi.shape
        M = Mt // nb
        N = M if syrk else Bhi.shape[1] // nb
        if syrk:
            Bhi, Blo = Ahi, Alo
        if M == 0 or N == 0 or KC == 0:                 # nothing to add
            return
        for t in (Ahi, Alo, Bhi, Blo):
            assert t.stride(2) == 1 and t.stride(1) == KC, "residue planes must have packed rows"
        _lib.call("sdpv_rns_gemm", self._h, _lib.ptr_strided(Ahi), _lib.ptr_strided(Alo), _lib.ptr_strided(Bhi),
                  _lib.ptr_strided(Blo), Ahi.stride(0), Bhi.stride(0), _lib.ptr(acc), acc.stride(1), g0, G, nb, M, N,
                  KC, (1 if syrk else 0) | (2 if fresh else 0) | (4 if unsigned else 0), _lib.stream())

    # ---- step 3: CRT of a block of entries (sdpvibe/rns.py:227-245)
    def crt_block(self, acc, N, j0, w, rows):
        """acc (n, rows_total, N) int16; block = all rows (< rows) x columns j0..j0+w ->
        (words (E/4, rows*w) int32, bit lengths (rows*w,) int64, rows*w)."""
        B = rows * w
        Wd = torch.empty((self.W, B), dtype=torch.int32, device=acc.device)
        bl = torch.empty((B,), dtype=torch.int64, device=acc.device)
        _lib.call("sdpv_crt_block", self._h, _lib.ptr(acc), acc.stride(0), N, j0, w, rows, _lib.ptr(Wd),
                  _lib.ptr(bl), _lib.stream())
        return Wd, bl, B

    def crt_norm(self, acc, N, j0, w, rows, rowexp, colexp, L, rows_per_block=None, pred=None):
        """CRT fused with MPF renormalisation: entry (r, jj) gets exponent
        rowexp[r] + colexp[r // rows_per_block, j0 + jj]; returns (m (L, rows*w), e (rows*w,)).
        pred (device int32 scalar): run only where it is nonzero (the outputs are undefined otherwise)."""
        B = rows * w
        O = torch.empty((L, B), dtype=torch.int32, device=acc.device)
        eO = torch.empty((B,), dtype=torch.int64, device=acc.device)
        args = (self._h, _lib.ptr(acc), acc.stride(0), N, j0, w, rows, rows_per_block or rows,
                _lib.ptr(rowexp.contiguous()), _lib.ptr(colexp.contiguous()), L, _lib.ptr(O), _lib.ptr(eO))
        if pred is None:
            _lib.call("sdpv_crt_norm", *args, _lib.stream())
        else:
            _lib.call("sdpv_crt_norm_if", *args, _lib.ptr(pred), _lib.stream())
        return O, eO


def plane_stride(nbytes):
    """Bytes between residue planes of consecutive moduli: nbytes rounded up to an odd multiple of 2 KB,
    so that planes of different moduli start on different HBM channels."""
    q = -(-nbytes // 2048)
    return 2048 * (q if q % 2 else q + 1)


def gemm_config(M, N, K):
    """Tile shapes of the reference's Triton kernels (sdpvibe/rns.py:38-54); kept for API
    compatibility.  The B200 kernel always uses 128 x 128 output tiles with 128-byte K slices."""
    return 128, 128, 128, 6
