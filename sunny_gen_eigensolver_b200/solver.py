"""Host-side mirror of the reference's Julia wrapper (SunnyGeneigBench.jl).

`Solver(n; device_id, bpb_request, tuning, cache, kernel)` -> `Solver(...)`
`run_kernel!(solver, H, S; W, U, info, stream)`             -> `run_kernel(...)`
`run_kernel!(solver, H, S, W, U, info; stream)`             -> `run_kernel(...)` with all buffers
`run_kernel_chunked!(solver, H, S, W, U, info, ns, chunk)` -> `run_kernel_chunked(...)`
plus `block_dim_x`, `batches_per_block`, `shared_mem_bytes`, `path_name`,
`kernel_mode`, `last_error`.

Buffers are torch CUDA tensors laid out exactly like the Julia arrays the
reference passes (column-major (n, n, batch)): a C-contiguous tensor of
shape (batch, n, n) whose [b, j, i] element is matrix b's entry (i, j).
`to_colmajor` / `from_colmajor` convert natural (batch, n, n) matrices.
Errors are raised as RuntimeError carrying the library's last_error text,
as the Julia wrapper raises `error(...)`.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Tuple

import torch

from . import _native as nat


def to_colmajor(M: torch.Tensor) -> torch.Tensor:
    """(batch, n, n) natural matrices -> column-major buffer layout."""
    return M.transpose(-1, -2).contiguous()


def from_colmajor(X: torch.Tensor) -> torch.Tensor:
    """column-major buffer layout -> natural (batch, n, n) matrices."""
    return X.transpose(-1, -2)


class Solver:
    """Owns one libsunny_geneig handle (SunnyGeneigBench.jl:37-57)."""

    def __init__(self, n: int, *, device_id: int = 0, bpb_request: int = 0, tuning: str = "suggested",
                 cache: str = "auto", kernel: str = "unified", regime: Optional[str] = None,
                 slots_per_sm: int = 0):
        """`regime` ("smem-cta", "smem-wide", "l2-slot") and `slots_per_sm` (1, 2)
        request an execution configuration through sunny_geneig_create_config;
        by default the library chooses by n."""
        L = nat.load()
        tuning_int = nat.TUNING_AUTOTUNE if tuning == "autotune" else nat.TUNING_SUGGESTED
        cache_int = {"nodisk": nat.CACHE_NODISK, "nocache": nat.CACHE_NOCACHE}.get(cache, nat.CACHE_AUTO)
        kernel_int = {"hybrid": nat.KERNEL_HYBRID, "mixed": nat.KERNEL_MIXED}.get(kernel, nat.KERNEL_UNIFIED)
        if regime or slots_per_sm:
            h = L.sunny_geneig_create_config(int(n), int(device_id), kernel_int,
                                             (regime or "").encode(), int(slots_per_sm))
            fn = "sunny_geneig_create_config"
        else:
            h = L.sunny_geneig_create_ex(int(n), int(device_id), int(bpb_request), tuning_int, cache_int,
                                         kernel_int)
            fn = "sunny_geneig_create_ex"
        if not h:
            raise RuntimeError(f"{fn} failed: {nat.last_error()}")
        self._lib = L
        self.handle = h
        self.n = int(n)
        self.kernel = kernel
        self.device_id = int(device_id)

    # ---- lifetime
    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.sunny_geneig_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- introspection (SunnyGeneigBench.jl:66-92)
    @property
    def block_dim_x(self) -> int:
        return self._lib.sunny_geneig_block_dim_x(self.handle)

    @property
    def batches_per_block(self) -> int:
        return self._lib.sunny_geneig_batches_per_block(self.handle)

    @property
    def shared_mem_bytes(self) -> int:
        return self._lib.sunny_geneig_shared_mem_bytes(self.handle)

    @property
    def path_name(self) -> str:
        return self._lib.sunny_geneig_path_name(self.handle).decode()

    @property
    def kernel_mode(self) -> str:
        v = self._lib.sunny_geneig_kernel_mode(self.handle)
        return {nat.KERNEL_HYBRID: "hybrid", nat.KERNEL_MIXED: "mixed"}.get(v, "unified")

    @property
    def regime(self) -> str:
        return self._lib.sunny_geneig_regime_name(self.handle).decode()

    # ---- solves
    def _check(self, H, S, W, U, info):
        n = self.n
        if H.dim() != 3 or H.shape[1] != n or H.shape[2] != n:
            raise ValueError(f"matrix size mismatch: solver.n={n}, H={tuple(H.shape)}")
        batch = H.shape[0]
        if tuple(S.shape) != (batch, n, n):
            raise ValueError("S size must match H")
        if tuple(W.shape) != (batch, n):
            raise ValueError("W must be (batch, n)")
        if tuple(U.shape) != (batch, n, n):
            raise ValueError("U must be (batch, n, n)")
        if tuple(info.shape) != (batch,):
            raise ValueError("info must be length batch")
        for t, dt in ((H, torch.complex128), (S, torch.complex128), (W, torch.float64),
                      (U, torch.complex128), (info, torch.int32)):
            if t.dtype != dt or not t.is_cuda or not t.is_contiguous():
                raise ValueError(f"buffers must be contiguous CUDA tensors of {dt}")
        return batch

    def launch(self, H, S, W, U, info, stream: Optional[torch.cuda.Stream] = None, stage: int = 4) -> None:
        batch = self._check(H, S, W, U, info)
        s = stream if stream is not None else torch.cuda.current_stream(H.device)
        if stage == 4:
            st = self._lib.sunny_geneig_launch(self.handle, H.data_ptr(), S.data_ptr(), W.data_ptr(),
                                               U.data_ptr(), info.data_ptr(), int(batch), s.cuda_stream)
        else:
            st = self._lib.sunny_geneig_launch_stage(self.handle, int(stage), H.data_ptr(), S.data_ptr(),
                                                     W.data_ptr(), U.data_ptr(), info.data_ptr(), int(batch),
                                                     s.cuda_stream)
        if st != nat.STATUS_OK:
            raise RuntimeError(f"sunny_geneig_launch failed (status={st}): {nat.last_error()}")

    def launch_sigma(self, S, W, U, info, stream: Optional[torch.cuda.Stream] = None) -> None:
        """Solves Sigma u = lambda S u with Sigma = diag(I_{n/2}, -I_{n/2}) (the spin-wave
        metric); H is implied and not read. Same output layouts as `launch`."""
        batch = self._check(S, S, W, U, info)
        s = stream if stream is not None else torch.cuda.current_stream(S.device)
        st = self._lib.sunny_geneig_launch_sigma(self.handle, S.data_ptr(), W.data_ptr(), U.data_ptr(),
                                                 info.data_ptr(), int(batch), s.cuda_stream)
        if st != nat.STATUS_OK:
            raise RuntimeError(f"sunny_geneig_launch_sigma failed (status={st}): {nat.last_error()}")

    def launch_sigma_intensity(self, S, O, qhat, energies, fwhm: float, W, spec, info,
                               stream: Optional[torch.cuda.Stream] = None) -> None:
        """The metric solve of `launch_sigma` reduced on the device to spin-wave
        intensities on an energy grid (sunny_geneig_launch_sigma_intensity):
        S (batch, n, n) column-major buffers, O (batch, n, 3) complex128 (the
        column-major 3 x n observable matrix per problem), qhat (batch, 3),
        energies (ne,), W (batch, n), spec (batch, ne) float64, info (batch,).
        U is never formed in memory."""
        batch = S.shape[0]
        n = self.n
        checks = ((S, (batch, n, n), torch.complex128), (O, (batch, n, 3), torch.complex128),
                  (qhat, (batch, 3), torch.float64), (W, (batch, n), torch.float64),
                  (info, (batch,), torch.int32))
        for t, shape, dt in checks:
            if tuple(t.shape) != shape or t.dtype != dt or not t.is_cuda or not t.is_contiguous():
                raise ValueError(f"expected a contiguous CUDA tensor {shape} of {dt}")
        ne = energies.shape[0]
        if (energies.dtype != torch.float64 or not energies.is_cuda or not energies.is_contiguous()
                or tuple(spec.shape) != (batch, ne) or spec.dtype != torch.float64 or not spec.is_contiguous()):
            raise ValueError("energies (ne,) and spec (batch, ne) must be contiguous float64 CUDA tensors")
        s = stream if stream is not None else torch.cuda.current_stream(S.device)
        st = self._lib.sunny_geneig_launch_sigma_intensity(
            self.handle, S.data_ptr(), O.data_ptr(), qhat.data_ptr(), energies.data_ptr(), int(ne), float(fwhm),
            W.data_ptr(), spec.data_ptr(), info.data_ptr(), int(batch), s.cuda_stream)
        if st != nat.STATUS_OK:
            raise RuntimeError(f"sunny_geneig_launch_sigma_intensity failed (status={st}): {nat.last_error()}")

    @staticmethod
    def _fourier_args(terms, q, batch):
        start, coef, disp = terms
        checks = ((start, None, torch.int32), (coef, None, torch.complex128), (disp, None, torch.float64),
                  (q, (batch, 3), torch.float64))
        for t, shape, dt in checks:
            if (t.dtype != dt or not t.is_cuda or not t.is_contiguous()
                    or (shape is not None and tuple(t.shape) != shape)):
                raise ValueError(f"fourier terms / q: expected contiguous CUDA tensors of {dt}")
        nt = coef.shape[0]
        if tuple(disp.shape) != (nt, 3):
            raise ValueError("disp must have shape (n_terms, 3)")
        return start.data_ptr(), coef.data_ptr(), disp.data_ptr(), int(nt), q.data_ptr()

    def device_terms(self, start, coef, disp, device=None):
        """Moves a packed term table (lswt.pack_terms) to the device."""
        dev = device if device is not None else torch.device("cuda", self.device_id)
        if start.shape[0] != self.n * self.n + 1:
            raise ValueError(f"start must have n*n + 1 = {self.n * self.n + 1} entries")
        return (torch.as_tensor(start, dtype=torch.int32).to(dev).contiguous(),
                torch.as_tensor(coef, dtype=torch.complex128).to(dev).contiguous(),
                torch.as_tensor(disp, dtype=torch.float64).reshape(-1, 3).to(dev).contiguous())

    def launch_fourier_sigma(self, terms, q, W, U, info, stream: Optional[torch.cuda.Stream] = None) -> None:
        """Metric solve with S(q) assembled on the device from Fourier terms
        (sunny_geneig_launch_fourier_sigma): terms = (start, coef, disp) from
        device_terms, q (batch, 3) float64; W (batch, n), U (batch, n, n)
        column-major, info (batch,) as for `launch`. S is never in memory."""
        batch = q.shape[0]
        n = self.n
        for t, shape, dt in ((W, (batch, n), torch.float64), (U, (batch, n, n), torch.complex128),
                             (info, (batch,), torch.int32)):
            if tuple(t.shape) != shape or t.dtype != dt or not t.is_cuda or not t.is_contiguous():
                raise ValueError(f"expected a contiguous CUDA tensor {shape} of {dt}")
        p_start, p_coef, p_disp, nt, p_q = self._fourier_args(terms, q, batch)
        s = stream if stream is not None else torch.cuda.current_stream(q.device)
        st = self._lib.sunny_geneig_launch_fourier_sigma(self.handle, p_start, p_coef, p_disp, nt, p_q,
                                                         W.data_ptr(), U.data_ptr(), info.data_ptr(), int(batch),
                                                         s.cuda_stream)
        if st != nat.STATUS_OK:
            raise RuntimeError(f"sunny_geneig_launch_fourier_sigma failed (status={st}): {nat.last_error()}")

    def launch_fourier_sigma_intensity(self, terms, q, O, qhat, energies, fwhm: float, W, spec, info,
                                       stream: Optional[torch.cuda.Stream] = None) -> None:
        """Assembly, metric solve and intensities in one launch
        (sunny_geneig_launch_fourier_sigma_intensity); the arguments after q
        are those of `launch_sigma_intensity`."""
        batch = q.shape[0]
        n = self.n
        checks = ((O, (batch, n, 3), torch.complex128), (qhat, (batch, 3), torch.float64),
                  (W, (batch, n), torch.float64), (info, (batch,), torch.int32))
        for t, shape, dt in checks:
            if tuple(t.shape) != shape or t.dtype != dt or not t.is_cuda or not t.is_contiguous():
                raise ValueError(f"expected a contiguous CUDA tensor {shape} of {dt}")
        ne = energies.shape[0]
        if (energies.dtype != torch.float64 or not energies.is_cuda or not energies.is_contiguous()
                or tuple(spec.shape) != (batch, ne) or spec.dtype != torch.float64 or not spec.is_contiguous()):
            raise ValueError("energies (ne,) and spec (batch, ne) must be contiguous float64 CUDA tensors")
        p_start, p_coef, p_disp, nt, p_q = self._fourier_args(terms, q, batch)
        s = stream if stream is not None else torch.cuda.current_stream(q.device)
        st = self._lib.sunny_geneig_launch_fourier_sigma_intensity(
            self.handle, p_start, p_coef, p_disp, nt, p_q, O.data_ptr(), qhat.data_ptr(), energies.data_ptr(),
            int(ne), float(fwhm), W.data_ptr(), spec.data_ptr(), info.data_ptr(), int(batch), s.cuda_stream)
        if st != nat.STATUS_OK:
            raise RuntimeError(
                f"sunny_geneig_launch_fourier_sigma_intensity failed (status={st}): {nat.last_error()}")

    def run_kernel(self, H: torch.Tensor, S: torch.Tensor, W: Optional[torch.Tensor] = None,
                   U: Optional[torch.Tensor] = None, info: Optional[torch.Tensor] = None,
                   stream: Optional[torch.cuda.Stream] = None) -> Tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
        """run_kernel! (SunnyGeneigBench.jl:104-133, 143-171): allocates any missing output."""
        batch, n = H.shape[0], self.n
        dev = H.device
        W = torch.zeros((batch, n), dtype=torch.float64, device=dev) if W is None else W
        U = torch.zeros((batch, n, n), dtype=torch.complex128, device=dev) if U is None else U
        info = torch.zeros((batch,), dtype=torch.int32, device=dev) if info is None else info
        self.launch(H, S, W, U, info, stream)
        return W, U, info

    def run_kernel_chunked(self, H, S, W, U, info, num_streams: int, chunk_size: int) -> None:
        """run_kernel_chunked! (SunnyGeneigBench.jl:191-251): round-robin chunks over
        `num_streams` streams with no inter-chunk synchronisation, joined at the end."""
        if num_streams < 1 or chunk_size < 1:
            raise ValueError("num_streams and chunk_size must be >= 1")
        batch = self._check(H, S, W, U, info)
        streams = [torch.cuda.Stream(H.device) for _ in range(num_streams)]
        cur = torch.cuda.current_stream(H.device)
        for s in streams:
            s.wait_stream(cur)
        off, k = 0, 0
        while off < batch:
            bs = min(chunk_size, batch - off)
            sl = slice(off, off + bs)
            self.launch(H[sl], S[sl], W[sl], U[sl], info[sl], streams[k % num_streams])
            off += bs
            k += 1
        for s in streams:
            s.synchronize()


def last_error() -> str:
    return nat.last_error()


class UnevenSolver:
    """Persistent solver for problems of up to 8 different sizes in one launch
    (sunny_geneig_uneven_*). `regimes[n]` is "smem-cta", "l2-slot" or None
    (the default choice by n); `per_item[n]` problems of size n make one work
    item (None: the library default). Buffers are dicts keyed by size, each
    in the column-major layout of `Solver.launch`."""

    REGIME_CODE = {None: 0, "smem-cta": 1, "l2-slot": 2}

    def __init__(self, sizes, regimes=None, per_item=None, device_id: int = 0):
        L = nat.load()
        self.sizes = [int(n) for n in sizes]
        k = len(self.sizes)
        regimes = regimes or {}
        per_item = per_item or {}
        arr = ctypes.c_int * k
        h = L.sunny_geneig_uneven_create(k, arr(*self.sizes),
                                         arr(*[self.REGIME_CODE[regimes.get(n)] for n in self.sizes]),
                                         arr(*[int(per_item.get(n) or 0) for n in self.sizes]), int(device_id))
        if not h:
            raise RuntimeError(f"sunny_geneig_uneven_create failed: {nat.last_error()}")
        self._lib, self.handle, self.device_id = L, h, int(device_id)

    @property
    def shape(self):
        """[(n, regime, problems per item)] in work order (descending n)."""
        k = len(self.sizes)
        ns, rs, ps = (ctypes.c_int * k)(), (ctypes.c_int * k)(), (ctypes.c_int * k)()
        m = self._lib.sunny_geneig_uneven_shape(self.handle, ns, rs, ps)
        return [(ns[i], "l2-slot" if rs[i] == 2 else "smem-cta", ps[i]) for i in range(m)]

    def launch(self, H, S, W, U, info, stream: Optional[torch.cuda.Stream] = None) -> None:
        k = len(self.sizes)
        ptr = lambda d: (ctypes.c_size_t * k)(*[d[n].data_ptr() if n in d else 0 for n in self.sizes])
        counts = (ctypes.c_int * k)(*[int(H[n].shape[0]) if n in H else 0 for n in self.sizes])
        dev = next(iter(H.values())).device
        s = stream if stream is not None else torch.cuda.current_stream(dev)
        st = self._lib.sunny_geneig_uneven_launch(self.handle, ptr(H), ptr(S), ptr(W), ptr(U), ptr(info), counts,
                                                  s.cuda_stream)
        if st != nat.STATUS_OK:
            raise RuntimeError(f"sunny_geneig_uneven_launch failed (status={st}): {nat.last_error()}")

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.sunny_geneig_uneven_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def solve(H: torch.Tensor, S: torch.Tensor, solver: Optional[Solver] = None,
          stage: int = 4) -> Tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
    """Natural-layout convenience: H, S (batch, n, n) CUDA complex128 matrices.
    Returns W (batch, n), U (batch, n, n) with U[b][:, k] the k-th eigenvector,
    and info (batch,), after the launch has completed."""
    n = H.shape[-1]
    own = solver is None
    solver = Solver(n, device_id=H.device.index or 0) if own else solver
    try:
        Hc, Sc = to_colmajor(H), to_colmajor(S)
        batch = H.shape[0]
        W = torch.zeros((batch, n), dtype=torch.float64, device=H.device)
        U = torch.zeros((batch, n, n), dtype=torch.complex128, device=H.device)
        info = torch.zeros((batch,), dtype=torch.int32, device=H.device)
        solver.launch(Hc, Sc, W, U, info, stage=stage)
        torch.cuda.synchronize(H.device)
        return W, from_colmajor(U), info
    finally:
        if own:
            solver.close()
