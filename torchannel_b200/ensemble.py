"""Ensembles of independent channels (uneven grids) on one or more GPUs.

Members are independent, so a multi-GPU ensemble shards them across ranks
(one process per GPU, members assigned round-robin) with no collective on the
hot path; the only collectives are host-side reductions of the timing and the
per-member diagnostics after the steps.

On one GPU there are two ways to advance the members:
* ``ChannelBatch`` (``Ensemble.batch``): every substep of every member is ONE
  persistent launch over the concatenated work of all members
  (``tc_batch_*``), two steps replayed as one CUDA graph;
  ``Ensemble.autotune_batch`` picks its shapes (CN rows per chunk, CTAs per
  SM) by timing them on the ensemble.
* per-member launches on per-member streams (``Ensemble.step``);
  ``Ensemble.capture`` records two steps of every member (forked onto the
  member streams) as one CUDA graph, and ``Ensemble.autotune`` picks each
  member's kernel shapes (Poisson path, CN chunk length).
"""
import ctypes

import numpy as np


def make_members(n=16, seed=0, sizes_xy=(64, 96, 128), sizes_z=(48, 64, 96), re_range=(2000.0, 5600.0),
                 gamma_range=(2.2, 2.8)):
    """Seeded member table: nx, ny from sizes_xy, nz from sizes_z, Re and
    gamma uniform in their ranges, one seed per member."""
    rng = np.random.default_rng(seed)
    out = []
    for m in range(n):
        out.append(dict(nx=int(rng.choice(sizes_xy)), ny=int(rng.choice(sizes_xy)), nz=int(rng.choice(sizes_z)),
                        Re=float(rng.uniform(*re_range)), gamma=float(rng.uniform(*gamma_range)),
                        seed=int(seed * 1000 + m)))
    return out


def partition(n_members, world, rank):
    """Member indices owned by `rank` (round-robin)."""
    return list(range(rank, n_members, world))


def aggregate(local_points, local_ms):
    """Whole-job throughput: sum of grid-point-steps over ranks / max-over-ranks
    time.  Uses the default process group when one is initialised."""
    import torch
    import torch.distributed as dist
    pts, ms = float(local_points), float(local_ms)
    if dist.is_available() and dist.is_initialized():
        dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
        t = torch.tensor([pts], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        m = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(m, op=dist.ReduceOp.MAX)
        pts, ms = float(t.item()), float(m.item())
    return pts / (ms / 1e3), pts, ms


class ChannelBatch:
    """Channels (one precision, one device; nx, ny in {64, 96, 128, 192,
    256}) stepped together: one persistent launch per substep for all of
    them (``tc_batch_step``).  Each member advances as ``Channel.step``
    would; its state, scalars and statistics stay on its own ``Channel``."""

    def __init__(self, channels):
        import torch
        from . import _lib as L
        self.L = L
        self.lib = L.lib()
        self.channels = list(channels)  # keeps the contexts alive
        n = len(self.channels)
        prec = self.channels[0]._desc.precision
        nb = ctypes.c_size_t()
        L.check(self.lib.tc_batch_table_bytes(n, prec, ctypes.byref(nb)))
        self._table = torch.empty(nb.value + 16, dtype=torch.uint8, device="cuda")
        base = (self._table.data_ptr() + 15) & ~15
        arr = (ctypes.c_void_p * n)(*[c.ctx.value for c in self.channels])
        b = ctypes.c_void_p()
        L.check(self.lib.tc_batch_create(arr, n, ctypes.c_void_p(base), nb.value, ctypes.byref(b)))
        self.b = b

    def __del__(self):
        try:
            if getattr(self, "b", None) is not None and self.b.value:
                import torch
                torch.cuda.synchronize()
                self.lib.tc_batch_destroy(self.b)
                self.b = None
        except Exception:
            pass

    def member_cn_rows(self, cn_rows=None):
        """CN rows per chunk each member uses under the shape's cn_rows
        (default: the current shape): the same for every member, its chunks
        fill the CN block's first warps."""
        L = cn_rows or self.info()["cn_rows"]
        return [L for _ in self.channels]

    def set_shape(self, cn_rows=16, ctas_per_sm=0):
        self.L.check(self.lib.tc_batch_set_shape(self.b, int(cn_rows), int(ctas_per_sm)))

    def use_graphs(self, on=True):
        self.L.check(self.lib.tc_batch_use_graphs(self.b, int(bool(on))))

    def step(self, scheme, dts, n_steps=1):
        import torch
        from .core import SCHEMES
        d = np.ascontiguousarray(np.broadcast_to(np.asarray(dts, dtype=np.float64), (len(self.channels),)))
        self.L.check(self.lib.tc_batch_step(self.b, SCHEMES[scheme] if isinstance(scheme, str) else int(scheme),
                                            d.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), int(n_steps),
                                            ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))

    def launches_per_step(self, scheme="IMEX"):
        """Kernel launches of one ensemble step: the RHS (one per 32 members
        with the tensor-copy tiles), the CN (IMEX: one per chunk count), the
        forward and inverse x transforms (one per transform length each), both
        y transforms and the z solve (one each) and the projection."""
        info = self.info()
        L = info["cn_rows"]
        chans = self.channels
        kb = 8 if chans[0]._desc.precision == self.L.TC_MIXED else 2  # planes of a tensor-copy tile
        tiles = sum(-(-c.nx // 32) * -(-c.ny // 8) * -(-c.nz // kb) for c in chans)
        rhs = -(-len(chans) // 32) if info["units"]["rhs"] == tiles else 1
        cn = len({-(-c.nz // L) for c in chans}) if scheme == "IMEX" else 0
        return rhs + cn + 3 + 2 * len({c.nx for c in chans}) + 1

    def info(self):
        shape, units, grids = (ctypes.c_int * 4)(), (ctypes.c_int * 7)(), (ctypes.c_int * 7)()
        self.L.check(self.lib.tc_batch_info(self.b, shape, units, grids))
        names = ["rhs", "cn", "fftx", "ffty", "tri", "ifftx", "proj"]
        return {"cn_rows": shape[0], "ctas_per_sm": shape[1], "built": bool(shape[2]), "cn_chunks": shape[3],
                "units": dict(zip(names, list(units))), "ctas": dict(zip(names, list(grids)))}


class Ensemble:
    """Members of an ensemble on the current GPU, each on its own stream."""

    def __init__(self, members, precision="mixed", Lx=4 * np.pi, Ly=4 * np.pi / 3, Lz=2.0):
        import torch
        from .core import Channel
        from .grid import generate_grid
        from .init import initialize_flow
        self.members = members
        self.channels, self.streams, self.dts = [], [], []
        for m in members:
            z_f, z_c, dz_f, dz_c = generate_grid(m["gamma"], m["nz"], Lz)
            s = torch.cuda.Stream()
            with torch.cuda.stream(s):
                ch = Channel(m["nx"], m["ny"], m["nz"], Lx, Ly, Lz, 1.0 / m["Re"], dz_f, dz_c, precision=precision)
                u, v, w, _ = initialize_flow(m["nx"], m["ny"], m["nz"], z_c, Ly, Lz, perturbation_intensity=0.1,
                                             seed=m["seed"])
                ch.set_state(u, v, w)
                ub = ch.bulk_velocity()
                ch.set_state(u * (1.0 / ub), v, w)
                ch.project_initial()
                dt = min(max(0.25 / ch.cfl_inverse(), 3e-4), 0.011)
            self.channels.append(ch)
            self.streams.append(s)
            self.dts.append(dt)

    def points(self):
        return sum(m["nx"] * m["ny"] * m["nz"] for m in self.members)

    def step(self, n_steps, concurrent=True):
        import torch
        if concurrent:
            for ch, s, dt in zip(self.channels, self.streams, self.dts):
                with torch.cuda.stream(s):
                    ch.step("IMEX", dt, n_steps)
        else:
            for ch, s, dt in zip(self.channels, self.streams, self.dts):
                with torch.cuda.stream(s):
                    ch.step("IMEX", dt, n_steps)
                s.synchronize()

    def synchronize(self):
        for s in self.streams:
            s.synchronize()

    # -- autotuning ------------------------------------------------------------
    def _save(self, ch):
        st = [t.clone() for t in ch.get_state()[:3]]
        try:
            hist = [t.clone() for t in ch.get_history()]
        except RuntimeError:  # no history yet (no step taken)
            hist = None
        return st, hist, float(ch.scalars[0].item())

    def _restore(self, ch, saved):
        st, hist, f = saved
        ch.set_state(*st, forcing=f)
        if hist is not None:
            ch.set_history(*hist)

    def autotune(self, steps=6, repeats=2):
        """For every member, time each candidate shape -- Poisson middle
        (three register-FFT kernels or the fused cluster kernel) x CN chunk
        length (16 or 32 rows) -- over `steps` steps (best of `repeats`), keep
        the fastest, and restore the member's state, history and forcing.
        Returns the chosen shapes and their step times (ms) per member."""
        import torch
        self.tuning = []
        for ch, s, dt, m in zip(self.channels, self.streams, self.dts, self.members):
            cands = []
            for fused in (False, True):
                for rows in (16, 32):
                    if rows == 16 and m["nz"] > 256:
                        continue
                    cands.append((fused, rows))
            best, times = None, {}
            with torch.cuda.stream(s):
                saved = self._save(ch)
                for fused, rows in cands:
                    try:
                        ch.use_fused_poisson(fused)
                    except RuntimeError:
                        continue  # cluster shape not schedulable here
                    ch.set_cn_chunk(rows)
                    ch.step("IMEX", dt, 2)  # history, tables and graphs of this shape
                    ms = []
                    for _ in range(repeats):
                        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                        e0.record(s)
                        ch.step("IMEX", dt, steps)
                        e1.record(s)
                        e1.synchronize()
                        ms.append(e0.elapsed_time(e1) / steps)
                    times[(fused, rows)] = min(ms)
                    self._restore(ch, saved)
                best = min(times, key=times.get)
                ch.use_fused_poisson(best[0])
                ch.set_cn_chunk(best[1])
                s.synchronize()
            self.tuning.append({"fused_poisson": best[0], "cn_rows": best[1],
                                "ms_per_step": {f"{'fused' if k[0] else '3k'}/cn{k[1]}": v for k, v in times.items()}})
        return self.tuning

    # -- one graph for the whole ensemble ------------------------------------------
    def capture(self):
        """Record two IMEX steps of every member, each on its own stream forked
        from and joined to one capture stream, as a single CUDA graph.  The
        members need their AB2 history (one eager step) first; two steps keep
        every member's buffer parity, so the graph can be replayed."""
        import torch
        for ch, s, dt in zip(self.channels, self.streams, self.dts):
            with torch.cuda.stream(s):
                ch.step("IMEX", dt, 1)  # history and CN tables in place
        torch.cuda.synchronize()
        main = torch.cuda.Stream()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=main):
            start = torch.cuda.Event()
            start.record(main)
            ends = []
            for ch, s, dt in zip(self.channels, self.streams, self.dts):
                s.wait_event(start)
                with torch.cuda.stream(s):
                    ch.step("IMEX", dt, 2)
                e = torch.cuda.Event()
                e.record(s)
                ends.append(e)
            for e in ends:
                main.wait_event(e)
        self.graph, self.graph_stream = g, main
        return g

    def step_graph(self, n_pairs):
        """Advance every member by 2 * n_pairs steps: n_pairs graph launches."""
        for _ in range(n_pairs):
            self.graph.replay()

    # -- one launch per substep for all members ----------------------------------
    def batch(self):
        """Group the members into a ChannelBatch (kept as ``self.batched``)."""
        import torch
        torch.cuda.synchronize()  # the members were set up on their own streams
        self.batched = ChannelBatch(self.channels)
        return self.batched

    def step_batch(self, n_steps, scheme="IMEX"):
        """Advance every member by n_steps with the ensemble launches (on the
        current stream)."""
        self.batched.step(scheme, self.dts, n_steps)

    def autotune_batch(self, steps=8, repeats=2, rows=(16, 32), ctas=(-1, 0, 2)):
        """Time every (CN rows per chunk, persistent CTAs per SM) shape of the
        ensemble launches over `steps` steps (best of `repeats`), keep the
        fastest, and restore every member's state, history and forcing.
        Returns the chosen shape and the step time (ms) of each candidate."""
        import torch
        b = self.batched
        saved = [self._save(ch) for ch in self.channels]
        deep = max(m["nz"] for m in self.members) > 256
        times = {}
        for r in rows:
            if r == 16 and deep:
                continue
            for c in ctas:
                b.set_shape(r, c)
                b.step("IMEX", self.dts, 2)  # tables, history and graph of this shape
                ms = []
                for _ in range(repeats):
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record()
                    b.step("IMEX", self.dts, steps)
                    e1.record()
                    e1.synchronize()
                    ms.append(e0.elapsed_time(e1) / steps)
                times[(r, c)] = min(ms)
                for ch, sv in zip(self.channels, saved):
                    self._restore(ch, sv)
        best = min(times, key=times.get)
        b.set_shape(*best)
        torch.cuda.synchronize()
        self.batch_tuning = {"cn_rows": best[0], "ctas_per_sm": best[1],
                             "ms_per_step": {f"cn{k[0]}/ctas{k[1]}": v for k, v in times.items()}}
        return self.batch_tuning

    def autotune_mode(self, steps=8, repeats=2):
        """Choose between the ensemble launches (tuned shape) and per-member
        launches on per-member streams (one graph, tuned member shapes): time
        both over `steps` steps and keep the faster as ``self.mode``
        ("batch" or "streams"), restoring every member's state.  Returns the
        two step times (ms)."""
        import torch
        saved = [self._save(ch) for ch in self.channels]
        if getattr(self, "batched", None) is None:
            self.batch()
        self.autotune_batch(steps=steps, repeats=repeats)
        times = {"batch": min(self.batch_tuning["ms_per_step"].values())}
        for ch, sv in zip(self.channels, saved):
            self._restore(ch, sv)
        self.autotune(steps=steps, repeats=repeats)
        self.capture()
        ms = []
        for _ in range(repeats):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            self.step_graph(max(1, steps // 2))
            e1.record()
            e1.synchronize()
            ms.append(e0.elapsed_time(e1) / (2 * max(1, steps // 2)))
        times["streams"] = min(ms)
        for ch, sv in zip(self.channels, saved):
            self._restore(ch, sv)
        torch.cuda.synchronize()
        self.mode = min(times, key=times.get)
        return times

    def diagnostics(self):
        import torch
        out = []
        for ch, s in zip(self.channels, self.streams):
            with torch.cuda.stream(s):
                out.append(ch.diagnostics())
        return out
