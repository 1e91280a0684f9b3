//go:build goav1_cuda

// decoder_postfilter_cuda.go - a FrameWorkPostFilterRunner backed by the B200
// post-filter library (libgoav1pf.so, C ABI in include/goav1pf.h).
//
// It belongs in the root of the goav1 module, next to
// decoder_postfilter_bind.go, and is compiled only with the goav1_cuda build
// tag, so the pure-Go module is unchanged.  Build with the library's header
// and shared object on the cgo paths:
//
//	CGO_CFLAGS=-I<this repository>/include \
//	CGO_LDFLAGS="-L<this repository>/goav1_b200 -Wl,-rpath,<this repository>/goav1_b200" \
//	go build -tags goav1_cuda ./...
//
// The runner mirrors decoderFrameWorkReusableSupportedPostFilterRunner
// (decoder_postfilter_bind.go:398-440): Apply runs the remaining supported
// stages of the frame in place and PostFilterOutput returns the film-grain
// display copy (decoder_postfilter_bind.go:252-256).  Side information is
// passed in goav1's own decode-time layouts; nothing is converted except the
// restoration unit records (packed into pf_lr_unit) and the CDEF noskip
// words (read through the handle's accessor).
//
// cgo pointer rules: the C structs handed to the library live in C memory
// (one allocation per runner), and every Go slice they point into is pinned
// with runtime.Pinner for the duration of the call; the library keeps no
// pointer after it returns (host frames are copied up and back inside it).
package goav1

/*
#cgo LDFLAGS: -lgoav1pf
#include <stdlib.h>
#include <string.h>
#include "goav1pf.h"
*/
import "C"

import (
	"errors"
	"fmt"
	"runtime"
	"unsafe"

	"github.com/thesyncim/goav1/internal/av1/cdef"
	internaldecoder "github.com/thesyncim/goav1/internal/av1/decoder"
	internalframe "github.com/thesyncim/goav1/internal/av1/frame"
	"github.com/thesyncim/goav1/internal/av1/loopfilter"
	"github.com/thesyncim/goav1/internal/av1/parser"
	"github.com/thesyncim/goav1/internal/av1/threading"
	internaltile "github.com/thesyncim/goav1/internal/av1/tile"
)

// ErrCUDAPostFilterDevice reports a failed device call (PF_ERR_DEVICE) or a
// missing device (PF_ERR_NO_DEVICE); ErrCUDAPostFilterTimeout a device wait
// that ran out (PF_ERR_TIMEOUT, only with a wait deadline).
var (
	ErrCUDAPostFilterDevice  = errors.New("goav1: CUDA post-filter device error")
	ErrCUDAPostFilterTimeout = errors.New("goav1: CUDA post-filter wait timed out")
)

// statusError maps a library status onto goav1's sentinel errors, so callers
// keep using errors.Is as with the Go runner (decoder.go:46-53).
func statusError(st C.int) error {
	switch st {
	case C.PF_OK:
		return nil
	case C.PF_ERR_INVALID_CDEF:
		return cdef.ErrInvalidCDEF
	case C.PF_ERR_INVALID_FILTER:
		return loopfilter.ErrInvalidFilter
	case C.PF_ERR_INVALID_PLAN:
		return internaltile.ErrInvalidPlan
	case C.PF_ERR_UNSUPPORTED:
		return ErrDecoderUnsupportedPostFilter
	case C.PF_ERR_SHORT_BUFFER:
		return internalframe.ErrShortBuffer
	case C.PF_ERR_INVALID_FORMAT:
		return internalframe.ErrInvalidFormat
	case C.PF_ERR_INVALID_BATCH:
		return threading.ErrInvalidBatch
	case C.PF_ERR_TIMEOUT:
		return ErrCUDAPostFilterTimeout
	case C.PF_ERR_INVALID_ARG:
		return internaldecoder.ErrInvalidFrameWorkState
	default:
		return fmt.Errorf("%w: %s: %s", ErrCUDAPostFilterDevice, C.GoString(C.pf_status_string(st)),
			C.GoString(C.pf_status_detail()))
	}
}

// cbool and cbool32 convert flags for the C structs (a binding of
// pf_lf_build's block record map would use them too).
func cbool(v bool) C.uint8_t {
	if v {
		return 1
	}
	return 0
}

func cbool32(v bool) C.int32_t {
	if v {
		return 1
	}
	return 0
}

// cudaPostFilterRunner is a FrameWorkPostFilterRunner on one CUDA device.
// Like the Go runner it is called once per completed frame from the decoder
// goroutine, never concurrently.
type cudaPostFilterRunner struct {
	ctx *C.pf_ctx

	// C-memory argument blocks, reused by every Apply.
	frame   *C.pf_frame
	disp    *C.pf_frame
	side    *C.pf_frame_side
	display internalframe.Frame // caller-owned display copy, valid until the next Apply
	dispBuf []byte
	grain   bool
	source  *internalframe.Frame

	noskip []byte       // 8 bytes per 64x64 CDEF unit
	units  [3][]C.pf_lr_unit
	pin    runtime.Pinner
}

// newCUDAPostFilterRunner opens the library on CUDA device `device`.
// waitTimeout > 0 bounds every device wait of a call (microseconds); 0 blocks.
func newCUDAPostFilterRunner(device int, waitTimeoutMicros int64) (*cudaPostFilterRunner, error) {
	var cfg C.pf_config
	cfg.device = C.int32_t(device)
	cfg.wait_timeout_us = C.int64_t(waitTimeoutMicros)
	var st C.int
	h := C.pf_create(&cfg, &st)
	if h == nil {
		return nil, statusError(st)
	}
	r := &cudaPostFilterRunner{ctx: h}
	r.frame = (*C.pf_frame)(C.calloc(1, C.size_t(unsafe.Sizeof(C.pf_frame{}))))
	r.disp = (*C.pf_frame)(C.calloc(1, C.size_t(unsafe.Sizeof(C.pf_frame{}))))
	r.side = (*C.pf_frame_side)(C.calloc(1, C.size_t(unsafe.Sizeof(C.pf_frame_side{}))))
	return r, nil
}

// Close releases the device context and the argument blocks.
func (r *cudaPostFilterRunner) Close() {
	if r == nil || r.ctx == nil {
		return
	}
	C.pf_destroy(r.ctx)
	C.free(unsafe.Pointer(r.frame))
	C.free(unsafe.Pointer(r.disp))
	C.free(unsafe.Pointer(r.side))
	r.ctx, r.frame, r.disp, r.side = nil, nil, nil, nil
}

// pinBytes pins a byte slice's backing array and returns its address (nil
// for an empty slice).
func (r *cudaPostFilterRunner) pinBytes(b []byte) unsafe.Pointer {
	if len(b) == 0 {
		return nil
	}
	r.pin.Pin(&b[0])
	return unsafe.Pointer(&b[0])
}

// setPlane fills one pf_plane from a frame plane (frame.Plane: Pix, Stride,
// Width, Height; the allocation is Stride/bps x len(Pix)/Stride samples).
func (r *cudaPostFilterRunner) setPlane(dst *C.pf_plane, p internalframe.Plane, bps int) {
	dst.data = r.pinBytes(p.Pix)
	dst.stride = C.int64_t(p.Stride)
	dst.width = C.int32_t(p.Width)
	dst.height = C.int32_t(p.Height)
	if p.Stride > 0 {
		dst.alloc_width = C.int32_t(p.Stride / bps)
		dst.alloc_height = C.int32_t(len(p.Pix) / p.Stride)
	}
}

// marshalFrame describes f (host memory) in dst; width and height are the
// coded luma size of the frame being filtered.
func (r *cudaPostFilterRunner) marshalFrame(dst *C.pf_frame, f *internalframe.Frame, width, height uint32) {
	C.memset(unsafe.Pointer(dst), 0, C.size_t(unsafe.Sizeof(*dst)))
	bps := f.Layout.BytesPerSample
	dst.width = C.int32_t(width)
	dst.height = C.int32_t(height)
	dst.bit_depth = C.uint8_t(f.Format.BitDepth)
	if f.Format.SubsamplingX {
		dst.ss_x = 1
	}
	if f.Format.SubsamplingY {
		dst.ss_y = 1
	}
	if f.Format.MonoChrome {
		dst.mono = 1
	}
	dst.memory = C.PF_MEM_HOST
	r.setPlane(&dst.plane[0], f.Y, bps)
	if !f.Format.MonoChrome {
		r.setPlane(&dst.plane[1], f.U, bps)
		r.setPlane(&dst.plane[2], f.V, bps)
	}
}

// stagesOf maps goav1's remaining post-filter stages onto PF_STAGE_* bits;
// a stage the library does not run (super-resolution goes through
// pf_frame_apply_superres, which this runner leaves to the Go path) is
// ErrDecoderUnsupportedPostFilter, as in the Go runner
// (decoder_postfilter_bind.go:277-282).
func stagesOf(ctx *internaldecoder.FrameWorkPostFilterContext) (C.uint32_t, error) {
	remaining := ctx.RemainingPostFilters()
	supported := internaldecoder.FrameWorkPostFilterLoopFilter | internaldecoder.FrameWorkPostFilterCDEF |
		internaldecoder.FrameWorkPostFilterLoopRestoration | internaldecoder.FrameWorkPostFilterFilmGrain
	if remaining&^supported != 0 {
		return 0, ErrDecoderUnsupportedPostFilter
	}
	var s C.uint32_t
	if remaining.Has(internaldecoder.FrameWorkPostFilterLoopFilter) {
		s |= C.PF_STAGE_LOOP_FILTER
	}
	if remaining.Has(internaldecoder.FrameWorkPostFilterCDEF) {
		s |= C.PF_STAGE_CDEF
	}
	if remaining.Has(internaldecoder.FrameWorkPostFilterLoopRestoration) {
		s |= C.PF_STAGE_LOOP_RESTORATION
	}
	if remaining.Has(internaldecoder.FrameWorkPostFilterFilmGrain) {
		s |= C.PF_STAGE_FILM_GRAIN
	}
	// The reference frame's padding is edge-replicated before film grain
	// when the frame refreshes a reference slot (postfilter.go:769-771).
	if ctx.Event.FrameSize.RefreshFrameFlags != 0 {
		s |= C.PF_STAGE_EXTEND_BORDERS
	}
	return s, nil
}

// marshalSide fills r.side from the context: stage bits, loop-filter levels
// with the decode-time masks and level cache (FrameWorkLoopFilterMasks),
// CDEF parameters with the unit index map and noskip words, the restoration
// frame parameters with every plane's unit records, and the film-grain
// parameters.  Every array the C struct points into is pinned.
func (r *cudaPostFilterRunner) marshalSide(ctx *internaldecoder.FrameWorkPostFilterContext) error {
	s := r.side
	C.memset(unsafe.Pointer(s), 0, C.size_t(unsafe.Sizeof(*s)))
	stages, err := stagesOf(ctx)
	if err != nil {
		return err
	}
	s.stages = stages
	s.side_memory = C.PF_MEM_HOST
	ev := &ctx.Event

	if stages&C.PF_STAGE_LOOP_FILTER != 0 {
		m := ctx.LoopFilterMasks
		if m == nil || !m.Valid() || len(m.Masks) == 0 || len(m.LevelCache) == 0 {
			// The decode-time masks are absent: the Go runner rebuilds them
			// from the record map (BuildFromMap); pf_lf_build does the same on
			// the device.  This runner expects the masks.
			return ErrDecoderUnsupportedPostFilter
		}
		lf := &s.lf
		lf.level_y[0] = C.uint8_t(ev.LoopFilter.LevelY[0])
		lf.level_y[1] = C.uint8_t(ev.LoopFilter.LevelY[1])
		lf.level_u = C.uint8_t(ev.LoopFilter.LevelU)
		lf.level_v = C.uint8_t(ev.LoopFilter.LevelV)
		lf.sharpness = C.uint8_t(ev.LoopFilter.Sharpness)
		r.pin.Pin(&m.Masks[0])
		lf.masks = (*C.uint16_t)(unsafe.Pointer(&m.Masks[0])) // lfmask.FilterMask: 640 uint16, Y then UV
		lf.sb128_w = C.int32_t(m.SB128W)
		lf.sb128_h = C.int32_t(m.SB128H)
		lf.level_cache = (*C.uint8_t)(r.pinBytes(m.LevelCache))
		lf.mi_cols = C.int32_t(m.Cols)
		lf.mi_rows = C.int32_t(m.Rows)
	}

	if stages&C.PF_STAGE_CDEF != 0 {
		p := ev.CDEF
		c := &s.cdef
		c.damping = C.uint8_t(p.Damping)
		c.bits = C.uint8_t(p.Bits)
		c.strength_count = C.uint8_t(p.StrengthCount)
		for i := 0; i < 8; i++ {
			c.y_strength[i] = C.uint8_t(p.YStrength[i])
			c.uv_strength[i] = C.uint8_t(p.UVStrength[i])
		}
		im := ctx.CDEFIndexMap
		if im == nil || len(im.Index) == 0 {
			return cdef.ErrInvalidCDEF
		}
		c.index = (*C.uint8_t)(r.pinBytes(im.Index))
		r.pin.Pin(&im.Read[0])
		c.read = (*C.uint8_t)(unsafe.Pointer(&im.Read[0])) // Go bools are single 0/1 bytes
		c.index_stride = C.int32_t(im.Stride)
		c.index_rows = C.int32_t(im.Rows)
		// Noskip words through the handle's accessor (the buffer itself is
		// unexported); without a bound grid every block is filtered.
		ucols, urows := int(im.Stride), int(im.Rows)
		if m := ctx.LoopFilterMasks; m != nil && m.NoSkipUnitGrid(ucols, urows) {
			if cap(r.noskip) < ucols*urows*8 {
				r.noskip = make([]byte, ucols*urows*8)
			}
			r.noskip = r.noskip[:ucols*urows*8]
			for uy := 0; uy < urows; uy++ {
				for ux := 0; ux < ucols; ux++ {
					w := m.NoSkipUnitMask(uy, ux)
					o := (uy*ucols + ux) * 8
					for b := 0; b < 8; b++ {
						r.noskip[o+b] = byte(w >> (8 * b))
					}
				}
			}
			c.noskip = (*C.uint8_t)(r.pinBytes(r.noskip))
		}
	}

	if stages&C.PF_STAGE_LOOP_RESTORATION != 0 {
		p := ev.Restoration
		lr := &s.lr
		for pl := 0; pl < 3; pl++ {
			lr._type[pl] = C.uint8_t(p.Type[pl])
		}
		lr.unit_size_y = C.uint16_t(p.UnitSizeY)
		lr.unit_size_uv = C.uint16_t(p.UnitSizeUV)
		rb := ctx.RestorationFrameBuffers
		if rb == nil {
			return internaltile.ErrInvalidPlan
		}
		for pl := 0; pl < 3; pl++ {
			recs := rb.Records[pl]
			if p.Type[pl] == parser.RestorationNone || len(recs) == 0 {
				continue
			}
			if cap(r.units[pl]) < len(recs) {
				r.units[pl] = make([]C.pf_lr_unit, len(recs))
			}
			u := r.units[pl][:len(recs)]
			for i := range u {
				u[i] = C.pf_lr_unit{}
			}
			for _, rec := range recs {
				if int(rec.Index) >= len(u) {
					return internaltile.ErrInvalidPlan
				}
				packLRUnit(&u[rec.Index], rec.Unit)
			}
			r.pin.Pin(&u[0])
			lr.units[pl] = &u[0]
			lr.unit_count[pl] = C.int32_t(len(u))
		}
	}

	if stages&C.PF_STAGE_FILM_GRAIN != 0 {
		packFilmGrain(&s.fg, ev.FilmGrain,
			ev.SequenceHeader.ColorConfig.MatrixCoefficients == parser.MatrixCoefficientsIdentity)
	}
	return nil
}

// packLRUnit stores one decoded restoration unit (tile.RestorationUnit):
// type, SGR parameter set and xqd, and taps 0..2 of the Wiener filters (the
// rest follow from symmetry, restoration/wiener.go:44-47).
func packLRUnit(dst *C.pf_lr_unit, u internaltile.RestorationUnit) {
	dst._type = C.uint8_t(u.Type)
	dst.sgr_set = C.uint8_t(u.SGRProj.ParamsIndex)
	dst.sgr_xqd[0] = C.int8_t(u.SGRProj.XQD[0])
	dst.sgr_xqd[1] = C.int8_t(u.SGRProj.XQD[1])
	for k := 0; k < 3; k++ {
		dst.wiener_v[k] = C.int8_t(u.Wiener.VFilter[k])
		dst.wiener_h[k] = C.int8_t(u.Wiener.HFilter[k])
	}
}

// packFilmGrain copies parser.FilmGrainParams (parser/film_grain.go:21-56)
// into pf_film_grain field by field.
func packFilmGrain(dst *C.pf_film_grain, g parser.FilmGrainParams, matrixIdentity bool) {
	b := cbool
	dst.apply = b(g.Apply)
	dst.chroma_scaling_from_luma = b(g.ChromaScalingFromLuma)
	dst.seed = C.uint16_t(g.Seed)
	dst.num_y_points = C.uint8_t(g.NumYPoints)
	for i := range g.YPoints {
		dst.y_points[i][0], dst.y_points[i][1] = C.uint8_t(g.YPoints[i][0]), C.uint8_t(g.YPoints[i][1])
	}
	dst.num_cb_points = C.uint8_t(g.NumCbPoints)
	dst.num_cr_points = C.uint8_t(g.NumCrPoints)
	for i := range g.CbPoints {
		dst.cb_points[i][0], dst.cb_points[i][1] = C.uint8_t(g.CbPoints[i][0]), C.uint8_t(g.CbPoints[i][1])
		dst.cr_points[i][0], dst.cr_points[i][1] = C.uint8_t(g.CrPoints[i][0]), C.uint8_t(g.CrPoints[i][1])
	}
	dst.scaling_shift = C.uint8_t(g.ScalingShift)
	dst.ar_coeff_lag = C.uint8_t(g.ARCoeffLag)
	for i := range g.ARCoeffsY {
		dst.ar_coeffs_y[i] = C.int8_t(g.ARCoeffsY[i])
	}
	for i := range g.ARCoeffsCb {
		dst.ar_coeffs_cb[i] = C.int8_t(g.ARCoeffsCb[i])
		dst.ar_coeffs_cr[i] = C.int8_t(g.ARCoeffsCr[i])
	}
	dst.ar_coeff_shift = C.uint8_t(g.ARCoeffShift)
	dst.grain_scale_shift = C.uint8_t(g.GrainScaleShift)
	dst.cb_mult, dst.cb_luma_mult, dst.cb_offset = C.uint8_t(g.CbMult), C.uint8_t(g.CbLumaMult), C.uint16_t(g.CbOffset)
	dst.cr_mult, dst.cr_luma_mult, dst.cr_offset = C.uint8_t(g.CrMult), C.uint8_t(g.CrLumaMult), C.uint16_t(g.CrOffset)
	dst.overlap = b(g.Overlap)
	dst.clip_to_restricted_range = b(g.ClipToRestrictedRange)
	dst.matrix_identity = b(matrixIdentity)
}

// ensureFrameLike makes r.display a frame of out's format, bound to a
// runner-owned buffer that grows only when a frame needs more
// (frame.RequiredSize / frame.Bind, frame/buffer.go:141-236).
func (r *cudaPostFilterRunner) ensureFrameLike(out *internalframe.Frame) error {
	layout, err := internalframe.RequiredSize(out.Format)
	if err != nil {
		return err
	}
	if cap(r.dispBuf) < layout.Size {
		r.dispBuf = make([]byte, layout.Size)
	}
	r.dispBuf = r.dispBuf[:layout.Size]
	d, err := internalframe.Bind(r.dispBuf, out.Format)
	if err != nil {
		return err
	}
	d.Color, d.Metadata = out.Color, out.Metadata
	r.display = d
	return nil
}

// Apply implements internaldecoder.FrameWorkPostFilterRunner: the remaining
// supported stages run on ctx.Output in place; with film grain the display
// frame is written into the runner's detached copy.
func (r *cudaPostFilterRunner) Apply(ctx internaldecoder.FrameWorkPostFilterContext) error {
	if r == nil || r.ctx == nil || ctx.Output == nil {
		return internaldecoder.ErrInvalidFrameWorkState
	}
	defer r.pin.Unpin()
	r.grain, r.source = false, nil
	if err := r.marshalSide(&ctx); err != nil {
		return err
	}
	out := ctx.Output
	r.marshalFrame(r.frame, out, ctx.Event.FrameSize.CodedWidth, ctx.Event.FrameSize.Height)
	var disp *C.pf_frame
	if r.side.stages&C.PF_STAGE_FILM_GRAIN != 0 && ctx.Event.FilmGrain.Apply {
		if err := r.ensureFrameLike(out); err != nil {
			return err
		}
		r.marshalFrame(r.disp, &r.display, ctx.Event.FrameSize.CodedWidth, ctx.Event.FrameSize.Height)
		disp = r.disp
		r.grain = true
	}
	if st := C.pf_frame_apply(r.ctx, r.frame, r.side, disp, nil); st != C.PF_OK {
		r.grain = false
		return statusError(st)
	}
	r.source = out
	return nil
}

// PostFilterOutput mirrors decoder_postfilter_bind.go:252-256 and :368-379:
// the grain display copy after a grain-applying Apply, else the filtered
// frame itself.
func (r *cudaPostFilterRunner) PostFilterOutput() (*Frame, bool) {
	if r == nil {
		return nil, false
	}
	if r.grain {
		return &r.display, true
	}
	if r.source != nil {
		return r.source, true
	}
	return nil, false
}

var (
	_ internaldecoder.FrameWorkPostFilterRunner = (*cudaPostFilterRunner)(nil)
	_ decoderFrameWorkPostFilterOutputProvider  = (*cudaPostFilterRunner)(nil)
)
