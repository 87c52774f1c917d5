"""Batched uneven mix on one B200: one graph-captured launch, autotuned.

A :class:`MixedBatch` collects

* Paillier fixed-exponent exponentiations ``out = base^e mod n^2`` of any
  key widths and batch sizes (each with its own key context and device
  buffers), run by one persistent work-stealing kernel per width
  (``cuhe_mix_*`` in ``include/cuhe_paillier.h``), and
* BFV NTT / INTT batches over device residue planes of rings of any degree
  (``cuhe_bfv_ntt`` in ``include/cuhe_bfv.h``),

and captures all of it in one CUDA graph: the Paillier kernels on the capture
stream, the NTT batches forked onto a second stream so that the two kinds
overlap, joined back before the graph ends.  ``replay()`` is then a single
launch from the host.

A width whose contexts select the FP64 pipe (n^2 of 4096 or 8192 bits by
default, ``PaillierDevice.set_fp64``) runs the persistent kernel of 52-bit-limb
products on that pipe, as those contexts' own calls do.  The autotuner picks,
per Paillier width, the (threads per instance, window) variant of the integer
kernel or, for those widths, the FP64 kernel, whichever finishes that width's
own batches fastest (and sets the contexts' pipe accordingly), and per ring
the (threads per CTA, radix) of its NTT batches, by timing the candidates on
the batch's own data with CUDA events.

``run_plain()`` is the comparison point: the same work as one launch per
operation with a wait after each (``PaillierDevice.modexp_array`` per batch,
one ``cuhe_bfv_ntt`` per NTT batch), using the same tuned variants.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Any

from cuhepy_b200 import _native
from cuhepy_b200._limbs import to_limbs, words_for


@dataclass
class _Modexp:
    ctx: Any
    base: Any
    out: Any
    count: int
    exponent: int


@dataclass
class _Ntt:
    ring: Any
    planes: Any
    primes: int
    inverse: bool
    original: Any


class MixedBatch:
    """See the module docstring."""

    def __init__(self, device: int = 0) -> None:
        import torch

        self._torch = torch
        self.device = int(device)
        self._lib = _native.paillier_lib()
        self._modexp: list[_Modexp] = []
        self._ntt: list[_Ntt] = []
        self.paillier_tuning: dict[int, tuple[int, int]] = {}
        self.paillier_fp64: dict[int, bool] = {}  # width -> FP64-pipe kernel chosen by the autotuner
        self.ntt_tuning: dict[int, tuple[int, int]] = {}  # id(ring) -> (threads, radix_log)
        self._mix = None
        self._graph = None
        self._side = torch.cuda.Stream(device=self.device)

    # -- building -------------------------------------------------------------
    def add_modexp(self, ctx, bases, exponent: int):
        """Queue ``bases[i]^exponent mod n^2`` for a device tensor of bases
        ([count, K] int32 limbs) under the context's key; returns the output
        tensor (filled when the batch runs)."""
        torch = self._torch
        if not (bases.is_cuda and bases.dim() == 2 and bases.shape[1] == ctx.words and bases.is_contiguous()):
            raise ValueError(f"bases must be a contiguous CUDA tensor [count, {ctx.words}]")
        out = torch.empty_like(bases)
        self._modexp.append(_Modexp(ctx, bases, out, int(bases.shape[0]), int(exponent)))
        self._invalidate()
        return out

    def add_ntt(self, ring, planes, primes: int, inverse: bool = False) -> None:
        """Queue an in-place NTT (or inverse) of device planes [count, N]."""
        self._ntt.append(_Ntt(ring, planes, int(primes), bool(inverse), planes.clone()))
        self._invalidate()

    def _invalidate(self) -> None:
        self._graph = None
        if self._mix is not None:
            self._lib.cuhe_mix_destroy(self._mix)
            self._mix = None

    def close(self) -> None:
        self._invalidate()

    def __del__(self) -> None:  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass

    # -- native plan ----------------------------------------------------------
    def _check(self, rc: int, mix=None) -> None:
        if rc == 0:
            return
        msg = self._lib.cuhe_mix_last_error(mix)
        text = msg.decode() if msg else str(rc)
        raise ValueError(text) if rc in (-1, -5) else RuntimeError(text)

    def _select_pipe(self, entries: list[_Modexp]) -> None:
        for e in entries:
            if e.ctx.words in self.paillier_fp64:
                e.ctx.set_fp64(1 if self.paillier_fp64[e.ctx.words] else 0)

    def _build_mix(self, entries: list[_Modexp], tuning: dict[int, tuple[int, int]]):
        self._select_pipe(entries)
        handle = ctypes.c_void_p()
        self._check(self._lib.cuhe_mix_create(self.device, ctypes.byref(handle)))
        mix = handle
        for e in entries:
            limbs = to_limbs([e.exponent], words_for(e.exponent))[0]
            self._check(self._lib.cuhe_mix_add_modexp(mix, e.ctx._ctx, e.base.data_ptr(), e.out.data_ptr(), e.count,
                                                       limbs.ctypes.data_as(_native.c_u32_p), limbs.size), mix)
        for words, (tpi, w) in tuning.items():
            self._check(self._lib.cuhe_mix_set_tuning(mix, words, tpi, w), mix)
        self._check(self._lib.cuhe_mix_plan(mix), mix)
        return mix

    def plan(self) -> None:
        if self._mix is None:
            self._mix = self._build_mix(self._modexp, self.paillier_tuning)

    def widths(self) -> list[dict]:
        self.plan()
        out = []
        for i in range(self._lib.cuhe_mix_widths(self._mix)):
            vals = [ctypes.c_int() for _ in range(4)]
            units, tasks = ctypes.c_int64(), ctypes.c_int()
            self._check(self._lib.cuhe_mix_info(self._mix, i, *(ctypes.byref(v) for v in vals), ctypes.byref(units),
                                                ctypes.byref(tasks)), self._mix)
            out.append({"words": vals[0].value, "threads_per_instance": vals[1].value, "window": vals[2].value,
                        "grid": vals[3].value, "units": units.value, "batches": tasks.value})
        return out

    # -- launching ------------------------------------------------------------
    def _ntt_launch(self, item: _Ntt, stream) -> None:
        from cuhepy_b200.bfv import _bfv_rns

        threads, radix = self.ntt_tuning.get(id(item.ring), (0, 0))
        _bfv_rns.ntt(item.ring, item.planes, item.primes, item.inverse, threads, radix, stream.cuda_stream)

    def launch(self, stream=None) -> None:
        """Enqueue the whole mix on `stream` (NTT batches forked to a side
        stream and joined back): no allocation, no synchronisation."""
        torch = self._torch
        self.plan()
        stream = stream or torch.cuda.current_stream(self.device)
        if self._ntt:
            fork = torch.cuda.Event()
            fork.record(stream)
            self._side.wait_event(fork)
        if self._modexp:
            self._check(self._lib.cuhe_mix_launch(self._mix, ctypes.c_void_p(stream.cuda_stream)), self._mix)
        if self._ntt:
            for item in self._ntt:
                self._ntt_launch(item, self._side)
            join = torch.cuda.Event()
            join.record(self._side)
            stream.wait_event(join)

    def capture(self):
        """Capture the mix in a CUDA graph (one launch per replay)."""
        torch = self._torch
        self.plan()
        stream = torch.cuda.Stream(device=self.device)
        # one eager run on the capture stream first (lazy module loading)
        with torch.cuda.stream(stream):
            self.launch(stream)
        stream.synchronize()
        self.restore_ntt_inputs()  # the NTT batches are in place
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=stream):
            self.launch(stream)
        self._graph = graph
        return graph

    def replay(self) -> None:
        if self._graph is None:
            self.capture()
        self._graph.replay()

    def check(self) -> None:
        """Wait for the device and raise on range errors of the last run."""
        self.plan()
        self._check(self._lib.cuhe_mix_check(self._mix), self._mix)

    def restore_ntt_inputs(self) -> None:
        for item in self._ntt:
            item.planes.copy_(item.original)

    # -- the comparison point -------------------------------------------------
    def run_plain(self) -> None:
        """One launch per operation, each waited for, same tuned variants."""
        torch = self._torch
        stream = torch.cuda.current_stream(self.device)
        self._select_pipe(self._modexp)
        for e in self._modexp:
            tpi, w = self.paillier_tuning.get(e.ctx.words, (0, 0))
            e.ctx.set_tuning(tpi, w)
            e.ctx.set_stream(stream.cuda_stream)
            e.ctx.modexp_array(e.base, e.exponent, e.out, e.count)
            stream.synchronize()
        for item in self._ntt:
            self._ntt_launch(item, stream)
            stream.synchronize()

    # -- autotuning -----------------------------------------------------------
    def _time(self, fn, reps: int) -> float:
        torch = self._torch
        stream = torch.cuda.current_stream(self.device)
        fn()  # warm
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(reps):
            fn()
        end.record(stream)
        end.synchronize()
        return start.elapsed_time(end) / reps

    def autotune(self, reps: int = 2) -> dict:
        """Pick the Paillier variant per width and the NTT launch shape per
        ring by timing them on this batch's own work; returns the timings."""
        from cuhepy_b200.paillier.gpu import PaillierDevice

        torch = self._torch
        report: dict[str, Any] = {"paillier": {}, "ntt": {}}
        stream = torch.cuda.current_stream(self.device)
        by_width: dict[int, list[_Modexp]] = {}
        for e in self._modexp:
            by_width.setdefault(e.ctx.words, []).append(e)
        for words, entries in sorted(by_width.items()):
            timings = {}
            self.paillier_fp64.pop(words, None)
            saved = [e.ctx.fp64 for e in entries]

            def timed(tuning):
                mix = self._build_mix(entries, tuning)
                try:
                    return self._time(
                        lambda: self._check(self._lib.cuhe_mix_launch(mix, ctypes.c_void_p(stream.cuda_stream)),
                                            mix), reps)
                finally:
                    self._lib.cuhe_mix_destroy(mix)

            try:
                for e in entries:
                    e.ctx.set_fp64(0)
                for tpi, w in PaillierDevice.VARIANTS[words]:
                    timings[(tpi, w)] = timed({words: (tpi, w)})
                if words >= 128:  # the FP64-pipe kernel's widths
                    for e in entries:
                        e.ctx.set_fp64(1)
                    timings["fp64"] = timed({})
            finally:
                for e, f in zip(entries, saved):
                    e.ctx.set_fp64(f)
            best = min(timings, key=timings.get)
            if words >= 128:
                self.paillier_fp64[words] = best == "fp64"
            if best == "fp64":
                self.paillier_tuning.pop(words, None)
            else:
                self.paillier_tuning[words] = best
            report["paillier"][words] = {"best": best, "ms": {(k if isinstance(k, str) else f"{k[0]}x{k[1]}"): v
                                                              for k, v in timings.items()}}
        rings: dict[int, list[_Ntt]] = {}
        for item in self._ntt:
            rings.setdefault(id(item.ring), []).append(item)
        for key, items in rings.items():
            n = items[0].ring.n
            candidates = []
            for threads in (n // 32, n // 16, n // 8):
                for radix in (2, 3, 4):
                    # radix 16 runs the register-heavy kernel: at most 512 threads
                    if 32 <= threads <= (512 if radix == 4 else 1024):
                        candidates.append((threads, radix))
            timings = {}
            for cand in candidates:
                self.ntt_tuning[key] = cand

                def run(items=items):
                    for it in items:
                        self._ntt_launch(it, stream)

                timings[cand] = self._time(run, reps)
            best = min(timings, key=timings.get)
            self.ntt_tuning[key] = best
            report["ntt"][n] = {"best": best, "ms": {f"{k[0]}t_r{1 << k[1]}": v for k, v in timings.items()}}
        self.restore_ntt_inputs()
        self._invalidate()
        return report
