"""Batched RGF: many independent selected inversions in one persistent launch.

The reference solves one matrix per ``rgf`` call
(``src/sinv/algorithms/rgf/rgf.py:17``); a transport code calls it once per
energy point A(E_k) = E_k I - H - Sigma(E_k).  ``rgf_batched`` takes the whole
list (each instance with its own block count and block size) and runs every
sweep inside one kernel launch, instances dispatched largest-first from a
device work queue.  ``BatchPlan`` keeps the outputs, workspace and uploaded
descriptors so repeated runs cost one memset and one launch (capturable in a
CUDA graph).
"""

import ctypes

import numpy as np

from .. import _lib
from . import _device as dev


class BatchPlan:
    """Outputs, workspace and descriptors of one batch, reusable across runs.

    ``instances``: sequence of ``(A_diag, A_upper, A_lower)`` (torch CUDA
    tensors or numpy arrays; one dtype for the batch, complex128 or float64).
    ``outputs`` (optional): matching ``(G_diag, G_upper, G_lower)`` tensors to
    write into instead of allocating.  ``inplace=True`` overwrites the input
    tensors with the results instead (torch CUDA inputs only; halves the
    memory, which lets a batch larger than half of HBM run as one launch).
    ``team="cta"`` runs every instance on a single CTA; by default large
    blocks get teams of 2-8 CTAs.

    ``workspace`` (optional): a device uint8 tensor to use instead of
    allocating one when it is large enough (``workspace_bytes``); plans that
    share one must run in order on one stream.

    ``schedule`` (optional): the team of every instance, the queue order and
    the int8 cut-over, as a dict {"team": [...], "priority": [...],
    "mixed_min_b": int} (any key may be left out); ``tune=True`` derives it
    from the autotuner's measured table for this GPU (``sinv_b200.autotune``,
    cached on disk; the first call for a block size measures it) and keeps
    the choice in ``self.schedule``.

    ``wait_limit`` (seconds, optional): bound of every device-side wait of
    this plan's launches (team barriers, scratch slots, streamed ready
    words; default 60 s).  An instance whose wait runs out gets status
    ``STATUS_TIMEOUT`` and is abandoned; the launch finishes the others.

    ``precision="mixed"`` (complex128 only) computes the block products of
    both sweeps on the int8 tensor cores (Ozaki splitting into ``digits``
    int8 slices, exact int32 accumulation, FP64 reconstruction) and keeps
    every block inverse in FP64.  ``digits`` 1..8 (default 7): each digit
    adds 7 bits to the operands and about two decimals to the result.  On
    tight-binding blocks (b = 512, eta = 1e-3) 6 digits give a
    selected-inverse error of 1.0e-8 against FP64 and 7 digits stay well
    below it.
    """

    def __init__(self, instances, sym_mat=False, save_off_diag=True, precision="fp64", outputs=None,
                 device=None, inplace=False, team=None, digits=7, workspace=None, wait_limit=None,
                 schedule=None, tune=False):
        torch = dev._torch()
        self.lib = _lib.load()
        if len(instances) == 0:
            raise ValueError("empty batch")
        tdt = dev.torch_dtype(instances[0][0])
        self.code = _lib.dtype_code(tdt)
        if self.code not in (_lib.C128, _lib.F64):
            raise TypeError("batched RGF takes complex128 or float64 instances")
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        self.flags = (_lib.SYM if sym_mat else 0) | (_lib.SAVE_OFFDIAG if save_off_diag else 0)
        if precision == "mixed":
            if self.code != _lib.C128:
                raise TypeError("mixed precision takes complex128 instances")
            if not 1 <= int(digits) <= 8:
                raise ValueError("digits must be in 1..8")
            self.flags |= _lib.PREC_MIXED | (int(digits) << _lib.PREC_DIGITS_SHIFT)
        if inplace:
            if not save_off_diag:
                raise ValueError("inplace requires save_off_diag=True")
            if not all(dev.is_torch(x) and x.is_cuda for x in instances[0] if x is not None):
                raise TypeError("inplace takes torch CUDA tensors")
            self.flags |= _lib.INPLACE
        if team == "cta":
            self.flags |= _lib.FORCE_CTA
        elif team is not None:
            raise ValueError("team must be None or 'cta'")
        self.save_off_diag = save_off_diag
        self.inputs, self.outputs, self.shapes = [], [], []
        descs = (_lib.BatchDesc * len(instances))()
        for k, inst in enumerate(instances):
            d, u, l = inst
            d = dev.to_device(d, tdt)
            n, b = int(d.shape[0]), int(d.shape[1])
            if d.dim() != 3 or d.shape[2] != b:
                raise ValueError("instance %d: A_diag must be (n, b, b)" % k)
            if n > 1:
                u = dev.to_device(u, tdt)
                l = dev.to_device(l, tdt)
                if tuple(u.shape) != (n - 1, b, b) or tuple(l.shape) != (n - 1, b, b):
                    raise ValueError("instance %d: off-diagonal blocks must be (%d, %d, %d)" % (k, n - 1, b, b))
            else:
                u = l = None
            if inplace:
                if n > 1 and (u.data_ptr() != inst[1].data_ptr() or l.data_ptr() != inst[2].data_ptr()) or \
                        d.data_ptr() != inst[0].data_ptr():
                    raise ValueError("inplace needs contiguous inputs of the batch dtype")
                Gd, Gu, Gl = d, u if u is not None else d[:0], l if l is not None else d[:0]
            elif outputs is not None:
                Gd, Gu, Gl = outputs[k]
            else:
                Gd = torch.empty((n, b, b), dtype=tdt, device=d.device)
                Gu = torch.empty((n - 1, b, b), dtype=tdt, device=d.device)
                Gl = torch.empty((n - 1, b, b), dtype=tdt, device=d.device)
            self.inputs.append((d, u, l))
            self.outputs.append((Gd, Gu, Gl))
            self.shapes.append((n, b))
            descs[k] = _lib.BatchDesc(d.data_ptr(), u.data_ptr() if u is not None else None,
                                      l.data_ptr() if l is not None else None, Gd.data_ptr(),
                                      Gu.data_ptr() if (save_off_diag and n > 1) else None,
                                      Gl.data_ptr() if (save_off_diag and n > 1) else None, n, b)
        self.descs = descs
        self.device = self.inputs[0][0].device
        if tune and schedule is None:
            from .. import autotune
            table = autotune.load_or_measure(sorted({b for _, b in self.shapes}), precision, int(digits),
                                             self.device)
            sms = torch.cuda.get_device_properties(self.device).multi_processor_count
            schedule = autotune.schedule(self.shapes, table, sms, precision)
        self.schedule = schedule
        self._sched = self._schedule_struct(schedule)
        nbytes = self.lib.sinvb_rgf_batched_sched_workspace_size(ctypes.cast(descs, ctypes.c_void_p), len(descs),
                                                                 self.code, self.flags, self._sched_ptr())
        with torch.cuda.device(self.device):
            if workspace is not None and workspace.numel() >= nbytes and workspace.data_ptr() % 256 == 0:
                self.ws = workspace  # shared with other plans run in order on one stream
            else:
                self.ws = dev.workspace(nbytes, self.device)
            self.status_dev = torch.zeros(len(descs), dtype=torch.int32, device=self.device)
        self.uploaded = False
        if wait_limit is not None:
            self.set_wait_limit(wait_limit)

    def set_wait_limit(self, seconds):
        """Bound (seconds) of every device wait of this plan's later launches."""
        _lib.check(self.lib.sinvb_rgf_batched_set_wait_limit(dev.ptr(self.ws), float(seconds)),
                   "sinvb_rgf_batched_set_wait_limit")

    def _schedule_struct(self, schedule):
        """ctypes sinvb_batch_schedule for `schedule` (None: no schedule)."""
        if schedule is None:
            return None
        count = len(self.shapes)
        st = _lib.BatchSchedule()
        self._sched_arrays = []
        if schedule.get("team") is not None:
            team = (ctypes.c_int * count)(*[int(t) for t in schedule["team"]])
            self._sched_arrays.append(team)
            st.team = ctypes.cast(team, ctypes.c_void_p)
        if schedule.get("priority") is not None:
            prio = (ctypes.c_float * count)(*[float(p) for p in schedule["priority"]])
            self._sched_arrays.append(prio)
            st.priority = ctypes.cast(prio, ctypes.c_void_p)
        st.mixed_min_b = int(schedule.get("mixed_min_b") or 0)
        return st

    def _sched_ptr(self):
        return ctypes.cast(ctypes.pointer(self._sched), ctypes.c_void_p) if self._sched is not None else None

    @staticmethod
    def workspace_bytes(shapes, dtype_code=None, flags=None, sym_mat=False, save_off_diag=True, precision="fp64",
                        inplace=False, digits=7):
        """Workspace bytes of a batch of (n, b) shapes (complex128 unless dtype_code)."""
        lib = _lib.load()
        code = _lib.C128 if dtype_code is None else dtype_code
        if flags is None:
            flags = (_lib.SYM if sym_mat else 0) | (_lib.SAVE_OFFDIAG if save_off_diag else 0)
            if precision == "mixed":
                flags |= _lib.PREC_MIXED | (int(digits) << _lib.PREC_DIGITS_SHIFT)
            if inplace:
                flags |= _lib.INPLACE
        descs = (_lib.BatchDesc * len(shapes))()
        for k, (n, b) in enumerate(shapes):
            descs[k] = _lib.BatchDesc(None, None, None, None, None, None, int(n), int(b))
        return int(lib.sinvb_rgf_batched_workspace_size(ctypes.cast(descs, ctypes.c_void_p), len(descs), code, flags))

    @property
    def count(self):
        return len(self.shapes)

    def run(self, stream=None):
        """Enqueue the batch (first run uploads descriptors, later runs only launch)."""
        torch = dev._torch()
        with torch.cuda.device(self.device):
            h = dev.stream_handle(stream)
            if not self.uploaded:
                fn = self.lib.sinvb_rgf_batched_sched_z if self.code == _lib.C128 else \
                    self.lib.sinvb_rgf_batched_sched_d
                rc = fn(ctypes.cast(self.descs, ctypes.c_void_p), len(self.descs), self.flags, self._sched_ptr(),
                        dev.ptr(self.ws), self.ws.numel(), dev.ptr(self.status_dev), h)
                _lib.check(rc, "sinvb_rgf_batched")
                self.uploaded = True
            else:
                fn = self.lib.sinvb_rgf_batched_rerun_z if self.code == _lib.C128 else \
                    self.lib.sinvb_rgf_batched_rerun_d
                _lib.check(fn(dev.ptr(self.ws), h), "sinvb_rgf_batched_rerun")

    def capture(self):
        """A ``torch.cuda.CUDAGraph`` holding one re-run of this batch (the
        workspace memsets and the persistent launch).  Replaying it recomputes
        every instance from the current contents of the input tensors; the
        first call uploads the descriptors outside the graph."""
        torch = dev._torch()
        with torch.cuda.device(self.device):
            if not self.uploaded:
                self.run()
            torch.cuda.synchronize(self.device)
            g = torch.cuda.CUDAGraph()
            s = torch.cuda.Stream(self.device)
            with torch.cuda.graph(g, stream=s):
                self.run(s)
            return g

    def run_streamed(self, ready, done, gen, stream=None):
        """Enqueue the batch so that instance k waits for ``ready[k] == gen``
        and raises ``done[k] = gen`` when finished (device int32 tensors of
        ``count`` words; see ``sinvb_rgf_batched_stream_z``).  Uploads the
        descriptors again on every call."""
        torch = dev._torch()
        with torch.cuda.device(self.device):
            if self._sched is not None:
                fn = (self.lib.sinvb_rgf_batched_stream_sched_z if self.code == _lib.C128
                      else self.lib.sinvb_rgf_batched_stream_sched_d)
                rc = fn(ctypes.cast(self.descs, ctypes.c_void_p), len(self.descs), self.flags, self._sched_ptr(),
                        dev.ptr(self.ws), self.ws.numel(), dev.ptr(self.status_dev), dev.ptr(ready), dev.ptr(done),
                        int(gen), dev.stream_handle(stream))
            else:
                fn = (self.lib.sinvb_rgf_batched_stream_z if self.code == _lib.C128
                      else self.lib.sinvb_rgf_batched_stream_d)
                rc = fn(ctypes.cast(self.descs, ctypes.c_void_p), len(self.descs), self.flags, dev.ptr(self.ws),
                        self.ws.numel(), dev.ptr(self.status_dev), dev.ptr(ready), dev.ptr(done), int(gen),
                        dev.stream_handle(stream))
            _lib.check(rc, "sinvb_rgf_batched_stream")
            self.uploaded = True

    def queue_order(self):
        """Instance indices in the order the kernel's queue hands them out:
        descending priority (the schedule's, as float32, else b^3 n), ties in
        instance order.  A streamed run copies its inputs in this order."""
        pr = (self.schedule or {}).get("priority") if isinstance(self.schedule, dict) else None
        if pr is not None:
            key = [float(np.float32(p)) for p in pr]
        else:
            key = [float(b) ** 3 * n for n, b in self.shapes]
        return sorted(range(len(self.shapes)), key=lambda k: -key[k])

    def statuses(self):
        """Per-instance device status (synchronises)."""
        return self.status_dev.cpu().numpy()

    def check(self):
        st = self.statuses()
        bad = np.nonzero(st)[0]
        if bad.size:
            k = int(bad[0])
            if st[k] == _lib.STATUS_PIVOT:
                raise np.linalg.LinAlgError(
                    "rgf_batched: zero or non-finite pivot in instance %d (%d instances failed)" % (k, bad.size))
            raise RuntimeError("rgf_batched: instance %d status %d" % (k, st[k]))

    def results(self, like=None):
        out = []
        for (Gd, Gu, Gl) in self.outputs:
            if not self.save_off_diag:
                Gu.fill_(float("nan"))
                Gl.fill_(float("nan"))
            if like is not None and not dev.is_torch(like):
                out.append((Gd.cpu().numpy(), Gu.cpu().numpy(), Gl.cpu().numpy()))
            else:
                out.append((Gd, Gu, Gl))
        return out


def rgf_batched(instances, sym_mat=False, save_off_diag=True, precision="fp64", check=True, stream=None,
                digits=7):
    """Selected inversion of every ``(A_diag, A_upper, A_lower)`` in ``instances``.

    Returns a list of ``(G_diag, G_upper, G_lower)`` in the input order, numpy
    when the inputs are numpy.  ``check`` synchronises and raises
    ``numpy.linalg.LinAlgError`` naming the first instance with a zero or
    non-finite pivot.
    """
    plan = BatchPlan(instances, sym_mat, save_off_diag, precision, digits=digits)
    plan.run(stream)
    if check:
        plan.check()
    return plan.results(like=instances[0][0])


def _available_bytes(torch, device):
    """Device bytes a new allocation can get: free memory plus the blocks
    torch's caching allocator holds but no tensor uses."""
    free, _ = torch.cuda.mem_get_info(device)
    return free + torch.cuda.memory_reserved(device) - torch.cuda.memory_allocated(device)


def rgf_batched_host(instances, outputs=None, sym_mat=False, precision="fp64", digits=7, wave_bytes=None,
                     device=None, check=True, schedule=None):
    """Selected inversion of host-resident instances streamed through the GPU.

    ``instances``: list of ``(A_diag, A_upper, A_lower)`` torch CPU tensors
    (complex128 or float64; pinned memory lets the copies overlap the
    compute).  ``outputs``: matching host tensors to receive
    ``(G_diag, G_upper, G_lower)``; may be the inputs themselves (results over
    the inputs); by default new host tensors.  Returns the outputs.

    The batch is cut into waves of at most ``wave_bytes`` of input (default: a
    third of the free device memory), in their given order.  Each wave runs as
    one persistent launch, in place in one of two device buffers, while the
    next wave's inputs copy in on one stream and the previous wave's results
    copy out on another, so PCIe traffic hides behind the sweeps.  Off-diagonal
    blocks are always computed.  ``schedule`` (when the batch fits as one
    launch): teams and queue order as for ``BatchPlan``, or ``"tune"`` for the
    autotuner's choice for a streamed batch (``autotune.stream_schedule``,
    from the measured table of this GPU); the inputs are copied in the
    queue's order.
    """
    torch = dev._torch()
    device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    if not instances:
        raise ValueError("empty batch")
    tdt = instances[0][0].dtype
    if wave_bytes is None:
        free = _available_bytes(torch, device)
        esize_ = 16 if tdt == torch.complex128 else 8
        total = sum((3 * int(d.shape[0]) - 2) * int(d.shape[1]) ** 2 for d, _, _ in instances) * esize_
        if total + (8 << 30) <= free:  # the whole batch fits: one launch, copies overlapping it
            return _host_one_launch(torch, instances, outputs, sym_mat, precision, digits, device, check,
                                    schedule)
    if tdt not in (torch.complex128, torch.float64):
        raise TypeError("rgf_batched_host takes complex128 or float64 host tensors")
    shapes = [(int(d.shape[0]), int(d.shape[1])) for d, _, _ in instances]
    elems = [(3 * n - 2) * b * b for n, b in shapes]
    esize = 16 if tdt == torch.complex128 else 8
    if outputs is None:
        outputs = [(torch.empty_like(d), torch.empty_like(u), torch.empty_like(l)) for d, u, l in instances]
    with torch.cuda.device(device):
        if wave_bytes is None:  # as few waves as fit: each wave waits for its longest chain
            free = _available_bytes(torch, device)
            wave_bytes = max(free // 3, max(elems) * esize)
        waves, cur, used = [], [], 0
        for k, e in enumerate(elems):
            if cur and (used + e) * esize > wave_bytes:
                waves.append(cur)
                cur, used = [], 0
            cur.append(k)
            used += e
        waves.append(cur)
        cap = max(sum(elems[k] for k in w) for w in waves)
        bufs = [torch.empty(cap, dtype=tdt, device=device) for _ in range(min(2, len(waves)))]
        ws_bytes = max(BatchPlan.workspace_bytes([shapes[k] for k in w], _lib.dtype_code(tdt), sym_mat=sym_mat,
                                                 precision=precision, inplace=True, digits=digits) for w in waves)
        ws = dev.workspace(ws_bytes, device)
        s_in, s_run, s_out = torch.cuda.Stream(device), torch.cuda.Stream(device), torch.cuda.Stream(device)
        out_done = [None] * len(waves)
        plans = []
        for wi, w in enumerate(waves):
            buf = bufs[wi % len(bufs)]
            views, off = [], 0
            for k in w:
                n, b = shapes[k]
                parts = []
                for rows in (n, n - 1, n - 1):
                    parts.append(buf[off:off + rows * b * b].view(rows, b, b))
                    off += rows * b * b
                views.append(tuple(parts))
            with torch.cuda.stream(s_in):
                if wi >= 2:
                    s_in.wait_event(out_done[wi - 2])  # the buffer's previous results are out
                for k, v in zip(w, views):
                    for dst, src in zip(v, instances[k]):
                        if dst.numel():
                            dst.copy_(src, non_blocking=True)
                ev_in = torch.cuda.Event()
                ev_in.record(s_in)
            s_run.wait_event(ev_in)
            with torch.cuda.stream(s_run):  # the plan's status array is cleared on the run stream
                plan = BatchPlan(views, sym_mat=sym_mat, precision=precision, inplace=True, digits=digits,
                                 workspace=ws)
            plan.run(s_run)
            ev_run = torch.cuda.Event()
            ev_run.record(s_run)
            plans.append(plan)
            with torch.cuda.stream(s_out):
                s_out.wait_event(ev_run)
                for k, v in zip(w, views):
                    for dst, src in zip(outputs[k], v):
                        if src.numel():
                            dst.copy_(src, non_blocking=True)
                out_done[wi] = torch.cuda.Event()
                out_done[wi].record(s_out)
        s_out.synchronize()
        s_run.synchronize()
        if check:
            for p in plans:
                p.check()
    return outputs


_gen_counter = [0]


def _host_one_launch(torch, instances, outputs, sym_mat, precision, digits, device, check, schedule=None):
    """rgf_batched_host when the whole batch fits on the device: one persistent
    launch whose teams wait for each instance's inputs (ready flags written
    after its copies) while the host copies them in, largest b^3 n first (the
    kernel's order); the host polls the done flags and copies each finished
    instance out while the launch runs on."""
    tdt = instances[0][0].dtype
    shapes = [(int(d.shape[0]), int(d.shape[1])) for d, _, _ in instances]
    if outputs is None:
        outputs = [(torch.empty_like(d), torch.empty_like(u), torch.empty_like(l)) for d, u, l in instances]
    if isinstance(schedule, str):
        if schedule != "tune":
            raise ValueError("schedule must be a dict, None or 'tune'")
        from .. import autotune
        table = autotune.load_or_measure(sorted({b for _, b in shapes}), precision, int(digits), device)
        sms = torch.cuda.get_device_properties(device).multi_processor_count
        schedule = autotune.stream_schedule(shapes, table, sms, precision, 16 if tdt == torch.complex128 else 8)
    _gen_counter[0] += 1
    gen = _gen_counter[0]
    with torch.cuda.device(device):
        buf = torch.empty(sum((3 * n - 2) * b * b for n, b in shapes), dtype=tdt, device=device)
        views, off = [None] * len(shapes), 0
        for k, (n, b) in enumerate(shapes):
            parts = []
            for rows in (n, n - 1, n - 1):
                parts.append(buf[off:off + rows * b * b].view(rows, b, b))
                off += rows * b * b
            views[k] = tuple(parts)
        count = len(shapes)
        ready = torch.zeros(count, dtype=torch.int32, device=device)
        done = torch.zeros(count, dtype=torch.int32, device=device)
        gen_host = torch.full((1,), gen, dtype=torch.int32).pin_memory()
        done_host = torch.zeros(count, dtype=torch.int32).pin_memory()
        s_in, s_run, s_out, s_poll = (torch.cuda.Stream(device) for _ in range(4))
        init = torch.cuda.Event()
        init.record(torch.cuda.current_stream(device))  # buffers and flag arrays allocated and zeroed
        for s_ in (s_in, s_run, s_out, s_poll):
            s_.wait_event(init)
        with torch.cuda.stream(s_run):
            plan = BatchPlan(views, sym_mat=sym_mat, precision=precision, inplace=True, digits=digits,
                             schedule=schedule)
        order = plan.queue_order()  # copy the inputs in the order the kernel's teams take them
        plan.run_streamed(ready, done, gen, s_run)
        with torch.cuda.stream(s_in):
            for k in order:
                for dst, src in zip(views[k], instances[k]):
                    if dst.numel():
                        dst.copy_(src, non_blocking=True)
                ready[k:k + 1].copy_(gen_host, non_blocking=True)
        issued = [False] * count
        left = count
        import time as _time
        t_start = _time.monotonic()
        while left:
            with torch.cuda.stream(s_poll):
                done_host.copy_(done, non_blocking=True)
            s_poll.synchronize()
            flags_now = done_host.numpy()
            kernel_over = s_run.query()
            for k in order:
                if not issued[k] and (flags_now[k] == gen or kernel_over):
                    with torch.cuda.stream(s_out):
                        for dst, src in zip(outputs[k], views[k]):
                            if src.numel():
                                dst.copy_(src, non_blocking=True)
                    issued[k] = True
                    left -= 1
            if left and _time.monotonic() - t_start > 3600:
                raise RuntimeError("rgf_batched_host: instances never finished")
            if left:
                _time.sleep(0.0005)
        s_out.synchronize()
        s_run.synchronize()
        if check:
            plan.check()
        del buf
    return outputs
