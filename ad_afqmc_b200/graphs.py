"""Energy blocks recorded as CUDA graphs.

``BlockGraph`` records one energy block of the phaseless loop for one walker
population — the body of ``sampler.propagate_phaseless`` with
``n_ene_blocks = n_sr_blocks = 1`` (sampling.py:52-94, 146-168, 343-365)
followed by the driver's ``e_estimate`` update (driver.py:168):

    pop_control_ene_shift = e_estimate ; n_killed = 0
    fields ~ N(0,1) (S, W, G)                  Philox, device-resident counter
    S x propagate_constrained                  Green's function reused across steps
    block end: QR, overlaps, local energies, clamp, block energy, pop-shift EMA
    zeta ~ U(0,1) ; comb reconfiguration ; overlaps of the new walkers
    e_estimate = 0.9 e_estimate + 0.1 E_block

Every per-block input lives on the device (RNG counter, zeta, scalars), so a
replay draws fresh random numbers and needs no host round trip.

``BatchGraph`` records the blocks of many independent solves (fragments of
different sizes) into ONE graph, each solve on its own forked stream, so a
single replay advances every fragment by one block and the solves overlap on
the device.
"""

from __future__ import annotations

import ctypes as C
from typing import List, Optional

import torch

from . import _lib
from .propagation import make_state, sync_scalars
from .walkers import UHFWalkers


class BlockGraph:
    def __init__(self, ham, ham_data, prop, trial, wave_data, prop_data, n_prop_steps: int = 10,
                 update_estimate: bool = True, reconfigure: bool = True, lno: bool = False,
                 external_fields: bool = False):
        """reconfigure=False leaves the comb (and the overlaps of the new
        walkers) out of the recorded block, for callers that reconfigure
        across ranks after each replay; update_estimate=False leaves out the
        e_estimate update (a caller with several ranks updates it from the
        all-reduced block energy).  lno=True records the block end of
        sampler_lno (sampling.py:586-631) for an rhf_lno trial and restricted
        walkers: block_out then holds (energy, weight, orbital energy).
        external_fields=True leaves the field draw out of the recorded block:
        the caller writes each block's fields into ``self.fields`` (S, W, G)
        before the replay (``HostFieldBlocks`` streams them from host memory);
        zeta still comes from the device stream."""
        self.prop, self.trial, self.wave_data, self.ham_data = prop, trial, wave_data, ham_data
        self.eng = prop.engine(ham_data, trial, wave_data)
        if not self.eng.has_prop:
            raise _lib.AfqError("propagation intermediates missing")
        self.S = int(n_prop_steps)
        self.update_estimate = update_estimate
        self.reconfigure = reconfigure
        self.pd = prop_data
        sync_scalars(prop_data)
        w = prop_data["walkers"]
        self.tensors = list(w.data) if isinstance(w, UHFWalkers) else [w.data]
        self.tmp = [torch.empty_like(t) for t in self.tensors]
        dev = self.tensors[0].device
        W = prop.n_walkers
        G = int(ham_data["chol"].shape[0])
        self.fields = torch.empty(self.S, W, G, dtype=torch.float64, device=dev)
        key = prop_data["key"]
        self.seed = key.seed
        self.counter = torch.tensor([key.counter], dtype=torch.int64, device=dev)
        self.zeta = torch.zeros(1, dtype=torch.float64, device=dev)
        self.lno = bool(lno)
        self.external_fields = bool(external_fields)
        self.block_out = torch.zeros(3 if self.lno else 2, dtype=torch.float64, device=dev)
        if self.lno:
            if isinstance(w, UHFWalkers) or "prjlo" not in wave_data:
                raise _lib.AfqError("the LNO block needs restricted walkers and wave_data['prjlo']")
            self.prj = torch.as_tensor(wave_data["prjlo"], dtype=torch.float64, device=dev).reshape(
                -1, trial.nelec[0]).contiguous()
            self.e_buf = torch.empty(W, dtype=torch.complex128, device=dev)
            self.o_buf = torch.empty(W, dtype=torch.complex128, device=dev)
        # device error flags of the recorded blocks, OR-ed over replays until check_status()
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        self.w_tmp = torch.empty_like(prop_data["weights"])
        self.idx = torch.empty(W, dtype=torch.int32, device=dev)
        self.small = torch.empty(W * 16, dtype=torch.float64, device=dev)  # own: solves may overlap
        self.mo = trial._mo_list(wave_data)
        self.graph: Optional[torch.cuda.CUDAGraph] = None
        self.launches_per_block = 0

    # -- the recorded body ---------------------------------------------------
    def body(self) -> None:
        n0 = _lib.launch_count()
        st = self.body_begin()
        self.body_steps(st)
        self.body_end(st)
        self.launches_per_block = _lib.launch_count() - n0

    def body_begin(self) -> _lib.afq_state:
        """The block's prologue: population shift, killed count, fields."""
        lib = _lib.lib()
        stream = _lib.stream_handle()
        sc = self.pd["_scalars"]
        sc[1].copy_(sc[0])  # pop_control_ene_shift = e_estimate
        sc[2].zero_()       # n_killed_walkers
        if not self.external_fields:
            _lib.check(lib.afq_normal_fields_dev(self.fields.data_ptr(), self.fields.numel(), self.seed,
                                                 self.counter.data_ptr(), stream), "afq_normal_fields_dev")
        return make_state(self.pd)  # GREEN_CURRENT clear: the first step computes G

    def body_steps(self, st: _lib.afq_state) -> None:
        lib = _lib.lib()
        stream = _lib.stream_handle()
        eng = self.eng
        p, w, wb = eng.handle
        for s in range(self.S):
            _lib.check(lib.afq_propagate_constrained(C.byref(eng.dims), p, C.byref(st),
                                                     self.fields[s].data_ptr(), w, wb, stream),
                       "afq_propagate_constrained")

    def body_end(self, st: _lib.afq_state) -> None:
        """Block end, reconfiguration, overlaps, e_estimate, status."""
        lib = _lib.lib()
        stream = _lib.stream_handle()
        pd, eng = self.pd, self.eng
        sc = pd["_scalars"]
        p, w, wb = eng.handle
        if self.lno:
            self._lno_block_end(lib, stream)
        else:
            _lib.check(lib.afq_block_end(C.byref(eng.dims), p, C.byref(st), self.block_out.data_ptr(),
                                         w, wb, stream), "afq_block_end")
        if not self.reconfigure:
            sc[2].div_(self.prop.n_walkers)
            if self.update_estimate:
                sc[0].mul_(0.9).add_(0.1 * self.block_out[0])
            self._fold_status()
            pd.pop("_afq_green_of", None)
            return
        _lib.check(lib.afq_uniform_dev(self.zeta.data_ptr(), self.seed, self.counter.data_ptr(), stream),
                   "afq_uniform_dev")
        win = _lib.pair(*[t.data_ptr() for t in self.tensors] + [None] * (2 - len(self.tensors)))
        wout = _lib.pair(*[t.data_ptr() for t in self.tmp] + [None] * (2 - len(self.tmp)))
        _lib.check(lib.afq_stochastic_reconfiguration_dev(
            C.byref(eng.dims), pd["weights"].data_ptr(), self.zeta.data_ptr(), _lib.AFQ_SR_LOCAL, win, wout,
            self.w_tmp.data_ptr(), self.idx.data_ptr(), stream), "afq_stochastic_reconfiguration_dev")
        for t, u in zip(self.tensors, self.tmp):
            t.copy_(u)
        pd["weights"].copy_(self.w_tmp)
        mo = _lib.pair(self.mo[0].data_ptr(), self.mo[-1].data_ptr())
        _lib.check(lib.afq_calc_overlap(C.byref(eng.dims), mo, win, pd["overlaps"].data_ptr(),
                                        self.small.data_ptr(), self.small.numel() * 8, stream),
                   "afq_calc_overlap")
        sc[2].div_(self.prop.n_walkers)
        if self.update_estimate:
            sc[0].mul_(0.9).add_(0.1 * self.block_out[0])
        self._fold_status()
        pd.pop("_afq_green_of", None)

    def _fold_status(self) -> None:
        """Move the engine's device error flag into self.status (device ops
        only, so it records into the graph)."""
        flag = self.eng.status_flag()
        torch.maximum(self.status, flag, out=self.status)
        flag.zero_()

    def check_status(self) -> None:
        """Raise AfqError if a device-side wait timed out in any block since
        the last check; reads (and clears) the recorded flag."""
        if int(self.status.item()) != 0:
            self.status.zero_()
            raise _lib.AfqError("a device-side wait timed out: the blocks since the last check are invalid")

    def _lno_block_end(self, lib, stream) -> None:
        """sampler_lno._block_scan after the steps (sampling.py:586-631): QR,
        overlaps, local and orbital energies on the propagator's engine, the
        reference's clamps against pop_control_ene_shift, block averages and
        the shift update; device work only, so it records into the graph."""
        pd, eng = self.pd, self.eng
        sc = pd["_scalars"]
        p, w, wb = eng.handle
        wts = pd["weights"]
        sc[2].add_(wts.numel() - torch.count_nonzero(wts).to(torch.float64))
        win = _lib.pair(self.tensors[0].data_ptr(), None)
        _lib.check(lib.afq_orthonormalize(C.byref(eng.dims), win, None, self.small.data_ptr(),
                                          self.small.numel() * 8, stream), "afq_orthonormalize")
        mo = _lib.pair(self.mo[0].data_ptr(), self.mo[-1].data_ptr())
        _lib.check(lib.afq_calc_overlap(C.byref(eng.dims), mo, win, pd["overlaps"].data_ptr(),
                                        self.small.data_ptr(), self.small.numel() * 8, stream),
                   "afq_calc_overlap")
        _lib.check(lib.afq_calc_energy(C.byref(eng.dims), p, win, self.e_buf.data_ptr(), w, wb, stream),
                   "afq_calc_energy")
        _lib.check(lib.afq_calc_orbenergy(C.byref(eng.dims), p, win, self.prj.data_ptr(),
                                          int(self.prj.shape[0]), self.o_buf.data_ptr(), w, wb, stream),
                   "afq_calc_orbenergy")
        lim = (2.0 / self.prop.dt) ** 0.5
        shift = sc[1].clone()
        e = torch.real(self.e_buf)
        e = torch.where(torch.abs(e - shift) > lim, shift, e)
        o = torch.where(torch.abs(e - shift) > lim, shift, torch.real(self.o_buf))
        bw = torch.sum(wts)
        self.block_out[0] = torch.sum(e * wts) / bw
        self.block_out[1] = bw
        self.block_out[2] = torch.sum(o * wts) / bw
        sc[1].copy_(0.9 * shift + 0.1 * self.block_out[0])

    # -- capture / replay ----------------------------------------------------
    def capture(self, warmup: int = 1, device_sync: bool = True) -> "BlockGraph":
        """Record the block.  With device_sync=False the capture runs on the
        current (non-default) stream without synchronising the device, so
        other streams keep running (used when admitting solves while others
        are in flight)."""
        if not device_sync:
            for _ in range(warmup):
                self.body()
            self.graph = torch.cuda.CUDAGraph()
            self.graph.capture_begin(capture_error_mode="thread_local")
            try:
                self.body()
            finally:
                self.graph.capture_end()
            return self
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            for _ in range(warmup):
                self.body()
        torch.cuda.current_stream().wait_stream(s)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.body()
        return self

    def replay(self) -> torch.Tensor:
        """One block; returns the block (energy, weight) device tensor."""
        self.graph.replay()
        return self.block_out

    @property
    def e_estimate(self) -> torch.Tensor:
        return self.pd["_scalars"][0]


class BatchGraph:
    """Blocks of many independent solves in one graph (one forked stream each)."""

    def __init__(self, blocks: List[BlockGraph], n_streams: int = 16):
        self.blocks = blocks
        self.n_streams = max(1, min(n_streams, len(blocks)))
        self.graph: Optional[torch.cuda.CUDAGraph] = None

    def _record(self):
        main = torch.cuda.current_stream()
        streams = [torch.cuda.Stream() for _ in range(self.n_streams)]
        for s in streams:
            s.wait_stream(main)
        for i, b in enumerate(self.blocks):
            with torch.cuda.stream(streams[i % self.n_streams]):
                b.body()
        for s in streams:
            main.wait_stream(s)

    def capture(self, warmup: int = 1) -> "BatchGraph":
        for _ in range(warmup):
            self._record()
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self._record()
        return self

    def replay(self) -> None:
        self.graph.replay()

    @property
    def launches_per_block(self) -> int:
        return sum(b.launches_per_block for b in self.blocks)


class GroupedBatchGraph:
    """Blocks of many independent mixed-precision solves in one graph, with
    the phaseless steps of all solves in grouped launches (afq_batch_*): per
    step each kernel family runs once for the whole batch, the force-bias,
    VHS and propagator contractions as persistent grouped tcgen05 kernels over
    (solve, tile) work lists.  The per-solve block prologue (fields) and block
    end (QR, energies, comb) run on forked streams as in ``BatchGraph``.  Each
    solve's results equal its own ``BlockGraph`` replays bit for bit.  At most
    64 solves (afq_batch limit); all with the same steps per block and Taylor
    terms."""

    def __init__(self, blocks: List[BlockGraph], n_streams: int = 16):
        if not 1 <= len(blocks) <= 64:
            raise _lib.AfqError("a grouped batch holds 1 to 64 solves")
        S = blocks[0].S
        for b in blocks:
            if b.S != S or b.external_fields or b.lno:
                raise _lib.AfqError("grouped batches need equal steps per block, device fields, no LNO")
            b.eng.ensure_workspace()
        self.blocks = blocks
        self.S = S
        self.n_streams = max(1, min(n_streams, len(blocks)))
        n = len(blocks)
        lib = _lib.lib()
        self._dims = (_lib.afq_dims * n)(*[b.eng.dims for b in blocks])
        self._prep = (C.c_void_p * n)(*[b.eng.prepared.data_ptr() for b in blocks])
        self._work = (C.c_void_p * n)(*[b.eng.work.data_ptr() for b in blocks])
        self._wbytes = (C.c_size_t * n)(*[b.eng.work_bytes for b in blocks])
        self._states = (_lib.afq_state * n)(*[make_state(b.pd) for b in blocks])
        self._fields = (C.c_void_p * n)(*[b.fields.data_ptr() for b in blocks])
        size = C.c_size_t()
        _lib.check(lib.afq_batch_table_size(n, C.cast(self._dims, C.c_void_p), C.byref(size)),
                   "afq_batch_table_size")
        dev = blocks[0].fields.device
        self.table = torch.empty((size.value + 511) // 8 + 64, dtype=torch.float64, device=dev)
        base = (self.table.data_ptr() + 255) & ~255
        self._handle = C.c_void_p()
        torch.cuda.synchronize()
        _lib.check(lib.afq_batch_create(n, C.cast(self._dims, C.c_void_p), C.cast(self._prep, C.c_void_p),
                                        C.cast(self._work, C.c_void_p), C.cast(self._wbytes, C.c_void_p),
                                        C.cast(self._states, C.c_void_p), C.cast(self._fields, C.c_void_p),
                                        base, size.value, C.byref(self._handle)), "afq_batch_create")
        self.graph: Optional[torch.cuda.CUDAGraph] = None
        self.launches_per_block = 0

    def _record(self):
        lib = _lib.lib()
        n0 = _lib.launch_count()
        main = torch.cuda.current_stream()
        streams = [torch.cuda.Stream() for _ in range(self.n_streams)]
        for s in streams:
            s.wait_stream(main)
        states = []
        for i, b in enumerate(self.blocks):
            with torch.cuda.stream(streams[i % self.n_streams]):
                states.append(b.body_begin())
        for s in streams:
            main.wait_stream(s)
        for step in range(self.S):
            _lib.check(lib.afq_batch_propagate_constrained(self._handle, step, 1 if step > 0 else 0,
                                                           _lib.stream_handle(main)),
                       "afq_batch_propagate_constrained")
        for s in streams:
            s.wait_stream(main)
        for i, b in enumerate(self.blocks):
            with torch.cuda.stream(streams[i % self.n_streams]):
                b.body_end(states[i])
        for s in streams:
            main.wait_stream(s)
        self.launches_per_block = _lib.launch_count() - n0

    def body(self) -> None:
        """One block, launched eagerly (no graph)."""
        self._record()

    def capture(self, warmup: int = 1) -> "GroupedBatchGraph":
        for _ in range(warmup):
            self._record()
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self._record()
        return self

    def replay(self) -> None:
        self.graph.replay()

    def check_status(self) -> None:
        for b in self.blocks:
            b.check_status()

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            try:
                _lib.lib().afq_batch_destroy(h)
            except Exception:
                pass
            self._handle = None


class HostFieldBlocks:
    """Blocks of a BlockGraph recorded with external_fields=True, fed from
    host memory: the fields of the next block are uploaded on a copy stream
    (into one of two device staging buffers) while the current block runs,
    then copied into the graph's field buffer just before its replay.  Each
    block's results (energy, weight and the walker weights) are read back to
    a pinned host buffer.

        runner = HostFieldBlocks(bg)
        runner.upload(fields_of_block_0)          # pinned (S, W, G) float64
        for b in range(n):
            out = runner.run(fields_of_block_b_plus_1)  # numpy (energy, weight, weights...)
    """

    def __init__(self, bg: BlockGraph):
        if not bg.external_fields or bg.graph is None:
            raise _lib.AfqError("HostFieldBlocks needs a captured BlockGraph with external_fields=True")
        self.bg = bg
        self.copy_stream = torch.cuda.Stream()
        self.staging = [torch.empty_like(bg.fields) for _ in range(2)]
        self.ready = [torch.cuda.Event() for _ in range(2)]
        self.free = [torch.cuda.Event() for _ in range(2)]
        self.n = 0
        self.uploaded = -1  # last block whose fields were queued
        W = bg.prop.n_walkers
        self.out_host = torch.empty(2 + W, dtype=torch.float64).pin_memory()
        self.status_host = torch.zeros(1, dtype=torch.int32).pin_memory()
        self.h2d_bytes = bg.fields.numel() * bg.fields.element_size()
        self.d2h_bytes = self.out_host.numel() * self.out_host.element_size()

    def upload(self, host_fields: torch.Tensor) -> None:
        """Queue the upload of the fields of block ``self.n`` (the next to run)."""
        self._upload(self.n, host_fields)

    def _upload(self, block: int, host_fields: torch.Tensor) -> None:
        i = block % 2
        if tuple(host_fields.shape) != tuple(self.bg.fields.shape):
            raise _lib.AfqError(f"fields must have shape {tuple(self.bg.fields.shape)}")
        if block != self.uploaded + 1:
            raise _lib.AfqError(f"fields of block {block} queued out of order (last queued: {self.uploaded})")
        self.uploaded = block
        with torch.cuda.stream(self.copy_stream):
            self.copy_stream.wait_event(self.free[i])  # the previous user of this buffer copied it out
            self.staging[i].copy_(host_fields, non_blocking=True)
            self.ready[i].record(self.copy_stream)

    def run(self, next_host_fields: Optional[torch.Tensor] = None):
        """Run block ``self.n`` (its fields must have been uploaded), queue
        the upload of the next block's fields, and return the block's
        (energy, weight) followed by the walker weights as a numpy array."""
        if self.uploaded < self.n:
            raise _lib.AfqError(f"the fields of block {self.n} were not uploaded")
        i = self.n % 2
        cur = torch.cuda.current_stream()
        cur.wait_event(self.ready[i])
        self.bg.fields.copy_(self.staging[i])
        self.free[i].record(cur)
        self.bg.replay()
        if next_host_fields is not None:
            self._upload(self.n + 1, next_host_fields)
        self.out_host[:2].copy_(self.bg.block_out[:2], non_blocking=True)
        self.out_host[2:].copy_(self.bg.pd["weights"], non_blocking=True)
        self.status_host.copy_(self.bg.status, non_blocking=True)
        cur.synchronize()
        self.n += 1
        if int(self.status_host[0]) != 0:
            self.bg.status.zero_()
            raise _lib.AfqError(f"block {self.n - 1}: a device-side wait timed out; its results are invalid")
        return self.out_host.numpy().copy()

