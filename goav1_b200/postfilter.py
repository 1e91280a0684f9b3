"""Host-side mirror of goav1's post-filter runner, over the C ABI.

PostFilterRunner mirrors decoderFrameWorkReusableSupportedPostFilterRunner
(decoder_postfilter_bind.go:398-440): apply() takes the frame and the
decode-time side information of one completed frame, leaves the frame as the
publishable reference (deblock, CDEF, loop restoration, border extension,
in place) and, when film grain applies, produces the display picture that
post_filter_output() returns (decoder_postfilter_bind.go:252-256, :434-439).
Errors are raised as the reference's sentinel errors (ErrInvalidCDEF,
ErrInvalidFilter, ErrInvalidPlan, ErrUnsupportedPostFilter, ErrShortBuffer).

DeviceFrame / device_side keep frames and side information resident in HBM
(torch tensors are used only as device allocations).
"""

import ctypes as C

import numpy as np

from . import abi, lib


class PostFilterError(Exception):
    code = None


class ErrInvalidCDEF(PostFilterError):
    code = abi.PF_ERR_INVALID_CDEF


class ErrInvalidFilter(PostFilterError):
    code = abi.PF_ERR_INVALID_FILTER


class ErrInvalidPlan(PostFilterError):
    code = abi.PF_ERR_INVALID_PLAN


class ErrUnsupportedPostFilter(PostFilterError):
    code = abi.PF_ERR_UNSUPPORTED


class ErrShortBuffer(PostFilterError):
    code = abi.PF_ERR_SHORT_BUFFER


class ErrInvalidFormat(PostFilterError):
    code = abi.PF_ERR_INVALID_FORMAT


class ErrInvalidArgument(PostFilterError):
    code = abi.PF_ERR_INVALID_ARG


class ErrDevice(PostFilterError):
    code = abi.PF_ERR_DEVICE


class ErrTimeout(PostFilterError):
    code = abi.PF_ERR_TIMEOUT


class ErrNoDevice(PostFilterError):
    code = abi.PF_ERR_NO_DEVICE


class ErrInvalidBatch(PostFilterError):
    code = abi.PF_ERR_INVALID_BATCH


_ERRORS = {cls.code: cls for cls in (ErrInvalidCDEF, ErrInvalidFilter, ErrInvalidPlan, ErrUnsupportedPostFilter,
                                     ErrShortBuffer, ErrInvalidFormat, ErrInvalidArgument, ErrDevice, ErrTimeout,
                                     ErrNoDevice, ErrInvalidBatch)}


def check(status):
    if status != abi.PF_OK:
        msg = lib().pf_status_string(status).decode()
        if status == abi.PF_ERR_DEVICE:
            msg += ": " + lib().pf_status_detail().decode()
        raise _ERRORS.get(status, PostFilterError)(msg)
    return status


def _nfb(w, h):
    """Number of 64x64 filter blocks over the MI grid of a w x h frame."""
    mi_cols, mi_rows = ((w + 7) >> 3) << 1, ((h + 7) >> 3) << 1
    return ((mi_cols + 15) // 16) * ((mi_rows + 15) // 16)


def validate(frame, side, display=None):
    """The status pf_frame_apply would return before touching anything."""
    return lib().pf_frame_validate(C.byref(frame), C.byref(side), C.byref(display) if display is not None else None)


class PostFilterRunner:
    """One post-filter runner per decoder; calls are serialised by the caller."""

    def __init__(self, device=0, timing=False, wait_timeout_us=0):
        L = lib()
        cfg = abi.pf_config(device=device, timing=1 if timing else 0, wait_timeout_us=wait_timeout_us)
        st = C.c_int(0)
        h = L.pf_create(C.byref(cfg), C.byref(st))
        if not h:
            check(st.value or abi.PF_ERR_NO_DEVICE)
        self._h = h
        self._display = None
        self.stats = abi.pf_stats()

    def apply(self, frame, side, display=None):
        """Runs side.stages on frame (in place) and grain into display."""
        st = lib().pf_frame_apply(self._h, C.byref(frame), C.byref(side),
                                  C.byref(display) if display is not None else None, C.byref(self.stats))
        check(st)
        self._display = display if (side.stages & abi.PF_STAGE_FILM_GRAIN) else None
        return self.stats

    @staticmethod
    def batch_items(items):
        """ctypes array of pf_batch_item from (frame, side, display) triples."""
        arr = (abi.pf_batch_item * len(items))()
        for i, (f, s, d) in enumerate(items):
            arr[i].frame = C.pointer(f)
            arr[i].side = C.pointer(s)
            arr[i].display = C.pointer(d) if d is not None else None
        return arr

    def apply_batch(self, items):
        """items: list of (frame, side, display) device-resident triples, or
        an array from batch_items()."""
        arr = items if isinstance(items, C.Array) else self.batch_items(items)
        check(lib().pf_batch_apply(self._h, arr, len(arr), C.byref(self.stats)))
        return self.stats

    def batch_graphs(self, enable=True):
        """Capture pf_batch_apply as CUDA graphs per batch signature."""
        check(lib().pf_batch_graphs(self._h, int(enable)))

    def set_persistent(self, group, ctas):
        """Persistent CTA count of a stage group (abi.PF_TUNE_*); 0 = one CTA per item."""
        check(lib().pf_set_persistent(self._h, group, ctas))

    def set_schedule(self, group, ctas=0, units_per_cta=1, staging=0, tile=0):
        """Schedule of a stage group (abi.PF_TUNE_*): persistent CTAs, work
        items per CTA, items prefetched ahead, deblocking tile shape."""
        s = abi.pf_schedule(ctas, units_per_cta, staging, tile)
        check(lib().pf_set_schedule(self._h, group, C.byref(s)))

    def set_frame_groups(self, groups):
        """1 or 2 frame groups per batch (two halves on two streams)."""
        check(lib().pf_set_frame_groups(self._h, groups))

    def get_schedule(self, group):
        s = abi.pf_schedule()
        check(lib().pf_get_schedule(self._h, group, C.byref(s)))
        return s

    def autotune(self, items, reps=3):
        """Searches each stage group's schedule on this batch (run in place:
        pass copies).  Returns pf_tune_result."""
        arr = items if isinstance(items, C.Array) else self.batch_items(items)
        out = abi.pf_tune_result()
        check(lib().pf_autotune(self._h, arr, len(arr), reps, C.byref(out)))
        return out

    def cdef_search(self, source, recon, noskip, qindex, lam, max_presets=8, damping=0, want_mse=True):
        """Encoder CDEF strength search (cdefSearcher.search + finish,
        internal/av1/encoder/cdef_search.go:580-945) on 8-bit 4:2:0 frames.
        Returns (pf_cdef_search_result, mse uint64[2, nfb, 64], fb_index uint8[nfb])."""
        nfb = _nfb(recon.width, recon.height)
        mse = np.empty((2, nfb, 64), np.uint64) if want_mse else None
        idx = np.empty(nfb, np.uint8)
        res = abi.pf_cdef_search_result()
        prm = abi.pf_cdef_search_params(qindex=qindex, damping=damping, max_presets=max_presets, lam=lam)
        ns = noskip.ctypes.data if noskip is not None else None
        check(lib().pf_cdef_search(self._h, C.byref(source), C.byref(recon), ns, C.byref(prm),
                                   mse.ctypes.data if want_mse else None, idx.ctypes.data, C.byref(res)))
        return res, mse, idx

    def cdef_search_ex(self, source, recon, noskip, qindex, lam, ctrls, max_presets=8, damping=0, want_mse=True):
        """cdef_search over an explicit trial list (abi.pf_cdef_search_ctrls,
        e.g. a picture plan's from cdef_plan_picture): any search level.
        Returns (pf_cdef_search_result, mse uint64[2, nfb, 64], fb_index)."""
        nfb = _nfb(recon.width, recon.height)
        mse = np.empty((2, nfb, 64), np.uint64) if want_mse else None
        idx = np.empty(nfb, np.uint8)
        res = abi.pf_cdef_search_result()
        prm = abi.pf_cdef_search_params(qindex=qindex, damping=damping, max_presets=max_presets, lam=lam)
        ns = noskip.ctypes.data if noskip is not None else None
        check(lib().pf_cdef_search_ex(self._h, C.byref(source), C.byref(recon), ns, C.byref(prm), C.byref(ctrls),
                                      mse.ctypes.data if want_mse else None, idx.ctypes.data, C.byref(res)))
        return res, mse, idx

    def cdef_apply(self, recon, noskip, qindex, result, fb_index, damping=0):
        """The encoder's CDEF application (cdefApplier.apply,
        internal/av1/encoder/cdef_apply.go:202-371): filters the 8-bit 4:2:0
        `recon` (pf_frame view, host or device) in place with a search's
        pf_cdef_search_result and per-block indices (uint8[nfb] or None), the
        units coded as the decoder rebuilds them from the noskip words."""
        prm = abi.pf_cdef_search_params(qindex=qindex, damping=damping, max_presets=8, lam=0.0)
        check(lib().pf_cdef_apply(self._h, C.byref(recon), noskip.ctypes.data if noskip is not None else None,
                                  C.byref(prm), C.byref(result),
                                  fb_index.ctypes.data if fb_index is not None else None))

    def apply_superres(self, coded, side, upscaled, display=None):
        """apply() for a super-resolved frame: deblock and CDEF on `coded`,
        the upscale, then restoration, border extension and grain on
        `upscaled` (grain into `display`)."""
        check(lib().pf_frame_apply_superres(self._h, C.byref(coded), C.byref(side), C.byref(upscaled),
                                            C.byref(display) if display is not None else None,
                                            C.byref(self.stats)))
        self._display = display if (side.stages & abi.PF_STAGE_FILM_GRAIN) else None
        return self.stats

    def apply_batch_superres(self, items):
        """pf_batch_apply_superres: items are (coded, side, upscaled, display)
        tuples (display may be None), all device or all host frames; the
        chain's stages run as batched launches over the frames."""
        arr = (abi.pf_superres_item * len(items))()
        for i, (c, s, u, d) in enumerate(items):
            arr[i].coded = C.pointer(c)
            arr[i].side = C.pointer(s)
            arr[i].up = C.pointer(u)
            arr[i].display = C.pointer(d) if d is not None else None
        check(lib().pf_batch_apply_superres(self._h, arr, len(arr), C.byref(self.stats)))
        return self.stats

    def superres_upscale(self, coded, upscaled):
        """The normative super-resolution upscale (superres.UpscalePlaneCoded,
        internal/av1/superres/superres.go:40-107) of every plane of `coded`
        (width = FrameSize.CodedWidth) into `upscaled` (width =
        FrameSize.UpscaledWidth); pf_frame views, both host or both device."""
        check(lib().pf_superres_upscale(self._h, C.byref(coded), C.byref(upscaled)))

    def lf_build(self, records, levels, ss_x=1, ss_y=1, mono=False, masks=None, level_cache=None):
        """Deblocking edge masks and level cache from the block record map:
        FrameWorkLoopFilterMasks.BuildFromMap
        (internal/av1/threading/loop_filter_masks.go:450-680) and
        populateLoopFilterLevelCacheFromMap
        (decoder/postfilter_loopfilter_masks.go:119-228), on the GPU.

        records: the map, a uint8/record array of shape (mi_rows, mi_cols)
        with dtype abi.lf_record_dtype(), or a torch CUDA tensor of shape
        (mi_rows, mi_cols, 32) uint8 (device resident).  levels: pf_lf_levels.
        With host records the outputs are numpy arrays (masks uint16
        [sb128_h*sb128_w, 640], level_cache uint8 [mi_rows, mi_cols, 4]);
        with device records they are torch CUDA tensors of those shapes
        (or the given `masks` / `level_cache` tensors)."""
        if hasattr(records, "data_ptr"):
            import torch

            rows, cols = records.shape[0], records.shape[1]
            sbw, sbh = (cols + 31) // 32, (rows + 31) // 32
            if masks is None:
                masks = torch.empty((sbh * sbw, abi.PF_LF_MASK_WORDS), dtype=torch.int16, device=records.device)
            if level_cache is None:
                level_cache = torch.empty((rows, cols, 4), dtype=torch.uint8, device=records.device)
            check(lib().pf_lf_build(self._h, records.data_ptr(), cols, rows, abi.PF_MEM_DEVICE, C.byref(levels),
                                    ss_x, ss_y, int(mono), masks.data_ptr(), level_cache.data_ptr(),
                                    abi.PF_MEM_DEVICE))
            return masks, level_cache
        rec = np.ascontiguousarray(records)
        rows, cols = rec.shape
        sbw, sbh = (cols + 31) // 32, (rows + 31) // 32
        masks = np.empty((sbh * sbw, abi.PF_LF_MASK_WORDS), np.uint16)
        level_cache = np.empty((rows, cols, 4), np.uint8)
        check(lib().pf_lf_build(self._h, rec.ctypes.data, cols, rows, abi.PF_MEM_HOST, C.byref(levels), ss_x, ss_y,
                                int(mono), masks.ctypes.data, level_cache.ctypes.data, abi.PF_MEM_HOST))
        return masks, level_cache

    def lr_search(self, source, recon, restored=None):
        """Encoder loop-restoration unit search on the luma of 8-bit 4:2:0
        frames: SearchWienerUnitU8 and SearchSGRProjUnitU8 per 64x64 unit
        (internal/av1/encoder/restoration.go:149-263) with the Wiener / SGRProj
        / none decision of EncodeLoopRestorationKeyframe
        (encoder/keyframe_lossy.go:2332-2383); with `restored`, its luma gets
        the decided filters applied (:2422-2453).  source, recon and restored
        are pf_frame views (all host or all device; restored may be recon).
        Returns the pf_lr_search_unit records in raster order."""
        horz, vert = abi.lr_unit_grid(recon.width, recon.height)
        units = (abi.pf_lr_search_unit * (horz * vert))()
        check(lib().pf_lr_search(self._h, C.byref(source), C.byref(recon),
                                 C.byref(restored) if restored is not None else None, units, horz * vert))
        return units

    def cdef_features(self, recon, noskip, qindex, damping=0):
        """Per-filter-block features (float32[nfb, 40]) of an 8-bit 4:2:0
        deblocked reconstruction, as the learned search computes them."""
        nfb = _nfb(recon.width, recon.height)
        X = np.zeros((nfb, abi.PF_MLP_FEATURES), np.float32)
        ns = noskip.ctypes.data if noskip is not None else None
        check(lib().pf_cdef_features(self._h, C.byref(recon), ns, qindex, damping, X.ctypes.data))
        return X

    def mlp_forward(self, model, X):
        """Softmax outputs float32[n, 128] (luma trials, then chroma trials)."""
        X = np.ascontiguousarray(X, np.float32)
        P = np.zeros((X.shape[0], abi.PF_MLP_OUTPUTS), np.float32)
        check(lib().pf_cdef_mlp_forward(self._h, C.byref(model), X.ctypes.data, X.shape[0], P.ctypes.data))
        return P

    def mlp_gradients(self, model, X, labels):
        """(mean loss, pf_cdef_mlp_grads) of the training kernels over one batch."""
        X = np.ascontiguousarray(X, np.float32)
        Y = np.ascontiguousarray(labels, np.uint8)
        loss = C.c_float()
        g = abi.pf_cdef_mlp_grads()
        check(lib().pf_cdef_mlp_gradients(self._h, C.byref(model), X.ctypes.data, Y.ctypes.data, X.shape[0],
                                          C.byref(loss), C.byref(g)))
        return loss.value, g

    def mlp_train(self, model, X, labels, epochs, batch=256, lr=2e-3, beta1=0.9, beta2=0.999, eps=1e-8,
                  weight_decay=1e-4, seed=1):
        """Adam training on the GPU, model updated in place; returns the
        per-epoch mean loss."""
        X = np.ascontiguousarray(X, np.float32)
        Y = np.ascontiguousarray(labels, np.uint8)
        prm = abi.pf_cdef_mlp_train_params(epochs=epochs, batch=batch, lr=lr, beta1=beta1, beta2=beta2, eps=eps,
                                           weight_decay=weight_decay, seed=seed)
        losses = np.zeros(epochs, np.float32)
        check(lib().pf_cdef_mlp_train(self._h, C.byref(model), X.ctypes.data, Y.ctypes.data, X.shape[0],
                                      C.byref(prm), losses.ctypes.data))
        return losses

    def cdef_search_learned(self, source, recon, noskip, qindex, lam, model, threshold=0.5, candidates=3,
                            max_presets=8, damping=0, want_mse=True, want_stats=True, refine=False):
        """The learned search: the network's top trials per block, all trials
        where it is unsure, then the reference's greedy selection (its
        refinement passes only with refine=True).  Returns
        (pf_cdef_search_result, mse uint64[2, nfb, 64], fb_index, pf_cdef_learned_stats)."""
        nfb = _nfb(recon.width, recon.height)
        mse = np.empty((2, nfb, 64), np.uint64) if want_mse else None
        idx = np.empty(nfb, np.uint8)
        res = abi.pf_cdef_search_result()
        st = abi.pf_cdef_learned_stats()
        prm = abi.pf_cdef_search_params(qindex=qindex, damping=damping, max_presets=max_presets, lam=lam)
        ns = noskip.ctypes.data if noskip is not None else None
        check(lib().pf_cdef_search_learned(self._h, C.byref(source), C.byref(recon), ns, C.byref(prm),
                                           C.byref(model), threshold, candidates,
                                           abi.PF_LEARNED_REFINE if refine else 0,
                                           mse.ctypes.data if want_mse else None, idx.ctypes.data,
                                           C.byref(res), C.byref(st) if want_stats else None))
        return res, mse, idx, st

    def post_filter_output(self):
        """(display frame, True) after a grain-applying apply(), else (None, False)."""
        return (self._display, self._display is not None)

    def sync(self):
        check(lib().pf_sync(self._h))

    @property
    def stream(self):
        return lib().pf_stream(self._h)

    def close(self):
        if getattr(self, "_h", None):
            lib().pf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Device residency helpers (torch tensors as plain device allocations).


class DeviceFrame:
    """A frame whose planes live in device memory, same geometry as a HostFrame."""

    def __init__(self, host, device="cuda"):
        import torch

        self.host = host
        dt = torch.uint8 if host.bit_depth == 8 else torch.int16
        self.tensors = []
        for p in host.planes:
            t = torch.empty(p.shape, dtype=dt, device=device)
            self.tensors.append(t)
        self.upload(host)

    def upload(self, host, non_blocking=False):
        import torch

        for t, p in zip(self.tensors, host.planes):
            src = torch.from_numpy(p.view(np.int16) if p.dtype == np.uint16 else p)
            t.copy_(src, non_blocking=non_blocking)

    def download(self, host=None):
        host = host or self.host.like()
        for t, p in zip(self.tensors, host.planes):
            a = t.cpu().numpy()
            p[:] = a.view(np.uint16) if p.dtype == np.uint16 else a
        return host

    def pf(self):
        bps = 1 if self.host.bit_depth == 8 else 2
        f = self.host.pf(memory=abi.PF_MEM_DEVICE, ptrs=[t.data_ptr() for t in self.tensors])
        for i, t in enumerate(self.tensors):
            f.plane[i].stride = t.stride(0) * bps
        return f

    def nbytes(self):
        return sum(t.numel() * t.element_size() for t in self.tensors)


def device_side(si, frame, device="cuda"):
    """Copy of a SideInfo (for HostFrame `frame`) whose arrays are device
    resident (side_memory=DEVICE)."""
    import torch

    s = abi.pf_frame_side()
    C.memmove(C.byref(s), C.byref(si.side), C.sizeof(s))
    s.side_memory = abi.PF_MEM_DEVICE
    keep = []

    def up(ptr, nbytes):
        if not ptr or nbytes == 0:
            return ptr
        buf = (C.c_uint8 * nbytes).from_address(ptr)
        t = torch.frombuffer(bytearray(buf), dtype=torch.uint8).to(device)
        keep.append(t)
        return t.data_ptr()

    lf = si.side.lf
    s.lf.masks = up(lf.masks, lf.sb128_w * lf.sb128_h * abi.PF_LF_MASK_WORDS * 2)
    s.lf.level_cache = up(lf.level_cache, 4 * lf.mi_cols * lf.mi_rows)
    cd = si.side.cdef
    n = cd.index_stride * cd.index_rows
    s.cdef.index = up(cd.index, n)
    s.cdef.read = up(cd.read, n)
    ucols, urows = (frame.width + 63) // 64, (frame.height + 63) // 64
    s.cdef.noskip = up(cd.noskip, ucols * urows * 8) if cd.noskip else None
    for p in range(3):
        if si.side.lr.units[p]:
            s.lr.units[p] = up(si.side.lr.units[p], si.side.lr.unit_count[p] * C.sizeof(abi.pf_lr_unit))
    from .synth import SideInfo

    return SideInfo(side=s, keep=keep + [si], blocks=si.blocks)


def cdef_plan_picture(level, islice, is_base=True, not_highest_layer=False, ref=None, ref_skip_percent=0):
    """A picture's CDEF plan at search level 1-8 (planSVTCDEF with the
    level's controls and updateOnRefInfo, internal/av1/encoder/cdef_frame.go:34-54):
    abi.pf_cdef_plan.  ref: the LAST reference's strengths
    (abi.pf_cdef_ref_strengths), needed by inter pictures at levels 5-8.
    Host logic only."""
    plan = abi.pf_cdef_plan()
    check(lib().pf_cdef_plan_picture(level, int(islice), int(is_base), int(not_highest_layer),
                                     C.byref(ref) if ref is not None else None, ref_skip_percent, C.byref(plan)))
    return plan


def cdef_search_level_rtc(islice, screen=False):
    """The search level goav1's real-time encoder uses (svtRTCCDEFSearchLevel)."""
    return lib().pf_cdef_search_level_rtc(int(islice), int(screen))
