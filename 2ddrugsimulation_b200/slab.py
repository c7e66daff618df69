"""Slab decomposition of a structured-grid tissue across GPUs.

The reference distributes a tissue by rows: PETSc splits A, B and V into
contiguous row ranges (MatCreateMPIAIJ with PETSC_DECIDE, fem.cpp:667-670),
MatMult and KSPSolve exchange ghost values and reduce the CG dot products
(fem.cpp:705-718), and each rank updates the cells of its own nodes
(heart.cpp:274-430). Here a part owns a contiguous range of grid planes
with its cells and its rows of A and B (csrc/slab.cu, cep_part_*); per CG
iteration the parts trade the boundary planes of the search direction with
their neighbours and gather every part's two partial sums, which each part
adds in part order. So every part stops at the same iteration and the
result is the same whichever rank holds which part.

The exchange is the caller's: `Links` moves planes and partials between the
parts of one process (aliased buffers, no copies) and, through
torch.distributed, between ranks (NCCL on GPUs; gloo for CPU parts). Ranks
hold equal numbers of contiguous parts. `SlabSolver` runs the split solve
over any parts that offer the cep_part operations (`DevicePart` here; the
oracle's CPU restatement in tests), and `SlabTissue` adds the Godunov
ionic step of each part's cells.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import Batch, _check, _dptr, lib

def split(n_planes: int, n_parts: int, part: int) -> tuple[int, int]:
    """(first plane, planes) of `part`: PETSC_DECIDE's rule, the first
    n_planes % n_parts parts one plane longer."""
    if not (1 <= n_parts <= n_planes and 0 <= part < n_parts):
        raise ValueError(f"cannot split {n_planes} planes into {n_parts} parts (part {part})")
    base, rem = divmod(n_planes, n_parts)
    return part * base + min(part, rem), base + (1 if part < rem else 0)


def rank_parts(n_parts: int, world: int, rank: int) -> range:
    """The contiguous parts rank `rank` holds (equal numbers per rank)."""
    if n_parts % world:
        raise ValueError(f"{n_parts} parts do not divide over {world} ranks")
    k = n_parts // world
    return range(rank * k, (rank + 1) * k)


def _addr(x) -> int | None:
    if x is None:
        return None
    if isinstance(x, int):
        return x
    return x.data_ptr()


class DevicePart:
    """One slab part on the current CUDA device (cep_part_*). Vectors are
    device tensors (float64) or device addresses."""

    def __init__(self, dim: int, nx: int, ny: int, nz: int, h: float, dt: float, D, part: int, n_parts: int,
                 stream=None):
        import torch
        nz = 1 if dim == 2 else nz
        n_elem = (nx - 1) * (ny - 1) * (nz - 1 if dim == 3 else 1)
        d = np.asarray(D, np.float64)
        d = np.ascontiguousarray(np.full((n_elem, 1), float(d)) if d.ndim == 0 else d.reshape(n_elem, -1))
        self.stream = torch.cuda.current_stream() if stream is None else stream
        h_ = ctypes.c_void_p()
        _check(lib().cep_part_create_grid(dim, nx, ny, nz, float(h), float(dt), _dptr(d), d.shape[1], part, n_parts,
                                           ctypes.c_void_p(self.stream.cuda_stream), ctypes.byref(h_)))
        self._h = h_
        r0, no, pl = ctypes.c_long(), ctypes.c_long(), ctypes.c_long()
        lo, hi = ctypes.c_int(), ctypes.c_int()
        _check(lib().cep_part_info(self._h, ctypes.byref(r0), ctypes.byref(no), ctypes.byref(pl), ctypes.byref(lo),
                                    ctypes.byref(hi)))
        self.index, self.n_parts, self.dim = part, n_parts, dim
        self.row0, self.n_own, self.plane = r0.value, no.value, pl.value
        self.has_lo, self.has_hi = bool(lo.value), bool(hi.value)

    def buffer(self, n: int):
        import torch
        return torch.zeros(n, dtype=torch.float64, device="cuda")

    def set_solver(self, rtol: float, max_iter: int = 10000, precond_norm: bool = True):
        _check(lib().cep_part_set_solver(self._h, float(rtol), int(max_iter), int(precond_norm)))

    def csr(self):
        """The owned rows (row_ptr, global columns, A, B)."""
        rp = np.zeros(self.n_own + 1, np.int32)
        cap = self.n_own * (27 if self.dim == 3 else 9)  # the stencil bounds the row length
        ci, av, bv = np.zeros(cap, np.int32), np.zeros(cap), np.zeros(cap)
        _check(lib().cep_part_get_csr(self._h, rp.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                       ci.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _dptr(av), _dptr(bv)))
        nnz = int(rp[-1])
        return rp, ci[:nnz], av[:nnz], bv[:nnz]

    def pack(self, v, lo, hi):
        _check(lib().cep_part_pack(self._h, _addr(v), _addr(lo), _addr(hi)))

    def cg_begin(self, v, v_lo, v_hi, partial):
        _check(lib().cep_part_cg_begin(self._h, _addr(v), _addr(v_lo), _addr(v_hi), _addr(partial)))

    def cg_direction(self, it: int, all_partials, send_lo, send_hi):
        _check(lib().cep_part_cg_direction(self._h, it, _addr(all_partials), self.n_parts, _addr(send_lo),
                                            _addr(send_hi)))

    def cg_product(self, it: int, p_lo, p_hi, partial):
        _check(lib().cep_part_cg_product(self._h, it, _addr(p_lo), _addr(p_hi), _addr(partial)))

    def cg_update(self, it: int, all_partials, partial):
        _check(lib().cep_part_cg_update(self._h, it, _addr(all_partials), self.n_parts, _addr(partial)))

    def cg_status(self, it: int) -> tuple[bool, int, float]:
        done, iters, res = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        _check(lib().cep_part_cg_status(self._h, it, ctypes.byref(done), ctypes.byref(iters), ctypes.byref(res)))
        return bool(done.value), iters.value, res.value

    def cg_end(self, v, t_new: float = 0.0):
        _check(lib().cep_part_cg_end(self._h, _addr(v), float(t_new)))

    def bind_cells(self, cells: Batch, s1_mask, bcl: float, t_crt: float, dur: float, n_pace: int,
                   act_thr: float = -30.0):
        m = None if s1_mask is None else np.ascontiguousarray(np.asarray(s1_mask, np.uint8).ravel())
        if m is not None and len(m) != self.n_own:
            raise ValueError(f"mask has {len(m)} entries, the part {self.n_own} rows")
        self._mask = m
        _check(lib().cep_part_bind_cells(self._h, cells._h, None if m is None else m.ctypes.data, float(bcl),
                                          float(t_crt), float(dur), int(n_pace), float(act_thr)))
        self.cells = cells

    def ionic_step(self, t: float):
        _check(lib().cep_part_ionic_step(self._h, float(t)))

    def activation(self) -> np.ndarray:
        out = np.zeros(self.n_own)
        _check(lib().cep_part_get_activation(self._h, _dptr(out)))
        return out

    def close(self):
        if getattr(self, "_h", None):
            _check(lib().cep_part_destroy(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Links:
    """Plane and partial-sum traffic of the parts this process holds
    (global indices parts[0].index .. parts[-1].index, contiguous), with
    torch.distributed carrying what crosses to the neighbouring ranks
    (`dist` None: every part is local)."""

    def __init__(self, parts, dist=None):
        self.parts, self.dist = parts, dist
        self.k0, self.n_parts = parts[0].index, parts[0].n_parts
        for j, p in enumerate(parts):
            if p.index != self.k0 + j or p.n_parts != self.n_parts:
                raise ValueError("a process holds contiguous parts of one split")
        if dist is None and len(parts) != self.n_parts:
            raise ValueError("without torch.distributed every part must be local")
        plane = parts[0].plane
        new = parts[0].buffer
        # up[j]: part j's upper boundary plane, read by part j + 1 as its lower
        # halo; down[j]: part j's lower boundary plane, read by part j - 1
        self.up = [new(plane) if p.has_hi else None for p in parts]
        self.down = [new(plane) if p.has_lo else None for p in parts]
        # halos that arrive from other ranks
        self.recv_lo = new(plane) if parts[0].has_lo else None
        self.recv_hi = new(plane) if parts[-1].has_hi else None
        self.all = new(2 * self.n_parts)
        self.local = new(2 * len(parts))

    def halo_lo(self, j):
        """The plane part j reads as its lower halo."""
        if not self.parts[j].has_lo:
            return None
        return self.up[j - 1] if j > 0 else self.recv_lo

    def halo_hi(self, j):
        if not self.parts[j].has_hi:
            return None
        return self.down[j + 1] if j + 1 < len(self.parts) else self.recv_hi

    def partial(self, j):
        """Where part j writes its two partial sums (never `all` itself:
        the parts of a phase still read the previous gather from it)."""
        return self.local[2 * j: 2 * j + 2]

    def exchange(self):
        """Deliver the boundary planes written into up / down to the
        neighbouring ranks."""
        if self.dist is None:
            return
        d, ops = self.dist, []
        rank = d.get_rank()
        first, last = self.parts[0], self.parts[-1]
        if first.has_lo:
            ops.append(d.P2POp(d.isend, self.down[0], rank - 1))
            ops.append(d.P2POp(d.irecv, self.recv_lo, rank - 1))
        if last.has_hi:
            ops.append(d.P2POp(d.isend, self.up[-1], rank + 1))
            ops.append(d.P2POp(d.irecv, self.recv_hi, rank + 1))
        if not ops:
            return
        if self.all.is_cuda:  # NCCL: one group, so the pairs cannot deadlock
            works = d.batch_isend_irecv(ops)
        else:
            works = [op.op(op.tensor, op.peer) for op in ops]
        for w in works:
            w.wait()

    def gather(self):
        """Every part's partials into `all`, in part order."""
        if self.dist is None:
            self.all.copy_(self.local)
            return
        d = self.dist
        chunks = [self.all[2 * len(self.parts) * r: 2 * len(self.parts) * (r + 1)] for r in range(d.get_world_size())]
        if self.all.is_cuda:
            d.all_gather_into_tensor(self.all, self.local)
        else:
            bufs = [c.clone() for c in chunks]
            d.all_gather(bufs, self.local)
            for c, b in zip(chunks, bufs):
                c.copy_(b)


class SlabSolver:
    """The split Jacobi-PCG over the parts this process holds."""

    def __init__(self, parts, dist=None, check_every: int = 8):
        self.parts = list(parts)
        self.links = Links(self.parts, dist)
        self.check_every = max(1, int(check_every))
        self.max_iter = 10000

    def set_solver(self, rtol: float, max_iter: int = 10000, precond_norm: bool = True):
        for p in self.parts:
            p.set_solver(rtol, max_iter, precond_norm)
        self.max_iter = int(max_iter)
        return self

    def solve(self, vs, t_new: float = 0.0) -> tuple[int, float]:
        """One implicit step A V = B V / dt in place on each part's V (vs[j]
        for the j-th local part). Returns (iterations, negative when
        max_iter was reached; relative residual)."""
        L, P = self.links, self.parts
        for j, p in enumerate(P):  # V's boundary planes to the neighbours
            p.pack(vs[j], L.down[j], L.up[j])
        L.exchange()
        for j, p in enumerate(P):
            p.cg_begin(vs[j], L.halo_lo(j), L.halo_hi(j), L.partial(j))
        L.gather()
        it = 0
        while True:
            for j, p in enumerate(P):
                p.cg_direction(it, L.all, L.down[j], L.up[j])
            if it % self.check_every == 0 or it >= self.max_iter:
                done, iters, res = P[0].cg_status(it)
                if done:
                    break
            L.exchange()
            for j, p in enumerate(P):
                p.cg_product(it, L.halo_lo(j), L.halo_hi(j), L.partial(j))
            L.gather()
            for j, p in enumerate(P):
                p.cg_update(it, L.all, L.partial(j))
            L.gather()
            it += 1
        for j, p in enumerate(P):
            p.cg_end(vs[j], t_new)
        return iters, res


class SlabTissue:
    """A Godunov tissue over slab parts: per step every part's ionic update
    at tissue time t, then the split diffusion solve (Cheart::processing,
    heart.cpp:127-165, on the rows of each part)."""

    def __init__(self, parts, cells, dt: float, dist=None, check_every: int = 8):
        self.parts, self.cells = list(parts), list(cells)
        self.solver = SlabSolver(self.parts, dist, check_every)
        self.dt, self.t, self.steps, self.iters = float(dt), 0.0, 0, []
        self._v = []
        for c in self.cells:
            ptr, ld = ctypes.c_void_p(), ctypes.c_long()
            _check(lib().cep_batch_device_states(c._h, ctypes.byref(ptr), ctypes.byref(ld)))
            self._v.append(ptr.value)  # row 0 of the SoA states: V

    def set_stimulus(self, masks, bcl: float, t_crt: float, dur: float, n_pace: int, act_thr: float = -30.0):
        for p, c, m in zip(self.parts, self.cells, masks):
            p.bind_cells(c, m, bcl, t_crt, dur, n_pace, act_thr)
        return self

    def run(self, n_steps: int):
        for _ in range(int(n_steps)):
            for p in self.parts:
                p.ionic_step(self.t)
            self.t += self.dt
            self.steps += 1
            self.iters.append(self.solver.solve(self._v, self.t)[0])
        return self
