//go:build goav1_cuda

// encoder_cdef_search_cuda.go - the encoder's CDEF strength search on the B200
// (libgoav1pf.so, pf_cdef_search_ex in include/goav1pf.h).
//
// It belongs in goav1's internal/av1/encoder package, next to
// cdef_search.go, and is compiled only with the goav1_cuda build tag (cgo
// paths as for decoder_postfilter_cuda.go).  cudaCDEFSearcher.search has the
// signature of cdefSearcher.search (cdef_search.go:580-634, with finish,
// :886-945), so the picture plan's decide step (cdef_frame.go:74) can call
// either: it takes the level's controls after updateOnRefInfo, searches
// every 64x64 filter block's listed trials on the device and returns the
// same CDEFParams and per-block indices.
package encoder

/*
#cgo LDFLAGS: -lgoav1pf
#include <stdlib.h>
#include <string.h>
#include "goav1pf.h"

// The argument block of one search call, in C memory.
typedef struct {
  pf_frame src, rec;
  pf_cdef_search_params params;
  pf_cdef_search_ctrls ctrls;
  pf_cdef_search_result result;
} goav1_cdef_search_args;
*/
import "C"

import (
	"errors"
	"fmt"
	"runtime"
	"unsafe"

	"github.com/thesyncim/goav1/internal/av1/threading"
)

// errCUDASearch reports a failed library call; the caller can fall back to
// the Go searcher.
var errCUDASearch = errors.New("encoder: CUDA CDEF search failed")

// cudaCDEFSearcher owns a device context and reusable argument storage.
// Like cdefSearcher it is used by one encoder goroutine at a time.
type cudaCDEFSearcher struct {
	ctx    *C.pf_ctx
	args   *C.goav1_cdef_search_args
	noskip []byte
	fbIdx  []uint8
	pin    runtime.Pinner
}

func newCUDACDEFSearcher(device int) (*cudaCDEFSearcher, error) {
	var cfg C.pf_config
	cfg.device = C.int32_t(device)
	var st C.int
	h := C.pf_create(&cfg, &st)
	if h == nil {
		return nil, fmt.Errorf("%w: %s", errCUDASearch, C.GoString(C.pf_status_string(st)))
	}
	a := (*C.goav1_cdef_search_args)(C.calloc(1, C.size_t(unsafe.Sizeof(C.goav1_cdef_search_args{}))))
	return &cudaCDEFSearcher{ctx: h, args: a}, nil
}

func (s *cudaCDEFSearcher) close() {
	if s == nil || s.ctx == nil {
		return
	}
	C.pf_destroy(s.ctx)
	C.free(unsafe.Pointer(s.args))
	s.ctx, s.args = nil, nil
}

// frame420 describes an 8-bit 4:2:0 SourceFrame420 (keyframe.go:27-31) as a
// host pf_frame; the chroma planes are (Width+1)/2 x (Height+1)/2.
func (s *cudaCDEFSearcher) frame420(dst *C.pf_frame, f *SourceFrame420) {
	C.memset(unsafe.Pointer(dst), 0, C.size_t(unsafe.Sizeof(*dst)))
	dst.width, dst.height = C.int32_t(f.Width), C.int32_t(f.Height)
	dst.bit_depth, dst.ss_x, dst.ss_y, dst.memory = 8, 1, 1, C.PF_MEM_HOST
	cw, ch := (f.Width+1)>>1, (f.Height+1)>>1
	planes := [3][]byte{f.Y, f.U, f.V}
	strides := [3]int{f.YStride, f.ChromaStride, f.ChromaStride}
	for p := 0; p < 3; p++ {
		w, h := f.Width, f.Height
		if p > 0 {
			w, h = cw, ch
		}
		s.pin.Pin(&planes[p][0])
		pl := &dst.plane[p]
		pl.data = unsafe.Pointer(&planes[p][0])
		pl.stride = C.int64_t(strides[p])
		pl.width, pl.height = C.int32_t(w), C.int32_t(h)
		pl.alloc_width = C.int32_t(strides[p])
		pl.alloc_height = C.int32_t(len(planes[p]) / strides[p])
	}
}

// noskipWords fills s.noskip with the 8-byte word of every 64x64 filter
// block (bit 8*by+bx: 8x8 block (by, bx) has a non-skip 4x4 MI cell), from
// the map's noskip grid or, without one, from its records as
// computeCDEFList does (cdef_search.go:410-447).
func (s *cudaCDEFSearcher) noskipWords(m *threading.FrameWorkLoopFilterMap, g cdefFrameGeometry) {
	n := g.nvfb * g.nhfb * 8
	if cap(s.noskip) < n {
		s.noskip = make([]byte, n)
	}
	s.noskip = s.noskip[:n]
	for fbr := 0; fbr < g.nvfb; fbr++ {
		for fbc := 0; fbc < g.nhfb; fbc++ {
			var word uint64
			if m.NoSkip != nil {
				word = m.NoSkip.UnitWord(fbr, fbc)
			} else {
				stride := int(m.Stride)
				nonSkip := func(r, c int) bool {
					if r >= int(m.Rows) || c >= stride {
						return false
					}
					rec := &m.Records[r*stride+c]
					return rec.Valid && !rec.SkipTransform
				}
				for r := 0; r < 16; r += 2 {
					for c := 0; c < 16; c += 2 {
						mr, mc := 16*fbr+r, 16*fbc+c
						if nonSkip(mr, mc) || nonSkip(mr, mc+1) || nonSkip(mr+1, mc) || nonSkip(mr+1, mc+1) {
							word |= 1 << uint((r>>1)*8+c>>1)
						}
					}
				}
			}
			o := (fbr*g.nhfb + fbc) * 8
			for b := 0; b < 8; b++ {
				s.noskip[o+b] = byte(word >> (8 * b))
			}
		}
	}
}

// search is cdefSearcher.search on the device: the controls' trial list
// (first pass, then second pass), chroma trials the level does not measure,
// the luma row subsampling and uvFromY go to pf_cdef_search_ex, whose
// greedy selection and RD choice are finish's.
func (s *cudaCDEFSearcher) search(src, recon *SourceFrame420, m *threading.FrameWorkLoopFilterMap,
	ctrls *svtCDEFSearchCtrls, qIndex uint8, lambda uint64) (svtCDEFDecision, error) {
	defer s.pin.Unpin()
	g := newCDEFFrameGeometry(recon.Width, recon.Height)
	a := s.args
	s.frame420(&a.src, src)
	s.frame420(&a.rec, recon)
	a.params = C.pf_cdef_search_params{qindex: C.int32_t(qIndex), damping: 0, max_presets: 8, lambda: C.double(lambda)}
	t := &a.ctrls
	C.memset(unsafe.Pointer(t), 0, C.size_t(unsafe.Sizeof(*t)))
	first := ctrls.firstPassFSNum
	total := first + ctrls.defaultSecondPassFSNum
	if total < 1 || total > C.PF_CDEF_MAX_TRIALS {
		return svtCDEFDecision{}, errCUDASearch
	}
	for gi := 0; gi < total; gi++ {
		if gi < first {
			t.y[gi], t.uv[gi] = C.int8_t(ctrls.defaultFirstPassFS[gi]), C.int8_t(ctrls.defaultFirstPassFSUV[gi])
		} else {
			t.y[gi] = C.int8_t(ctrls.defaultSecondPassFS[gi-first])
			t.uv[gi] = C.int8_t(ctrls.defaultSecondPassFSUV[gi-first])
		}
	}
	t.count = C.int32_t(total)
	t.subsampling = C.int32_t(ctrls.subsamplingFactor)
	if ctrls.uvFromY {
		t.uv_from_y = 1
	}
	s.noskipWords(m, g)
	nfb := g.nvfb * g.nhfb
	if cap(s.fbIdx) < nfb {
		s.fbIdx = make([]uint8, nfb)
	}
	s.fbIdx = s.fbIdx[:nfb]
	s.pin.Pin(&s.noskip[0])
	s.pin.Pin(&s.fbIdx[0])
	st := C.pf_cdef_search_ex(s.ctx, &a.src, &a.rec, (*C.uint8_t)(unsafe.Pointer(&s.noskip[0])), &a.params, t, nil,
		(*C.uint8_t)(unsafe.Pointer(&s.fbIdx[0])), &a.result)
	if st != C.PF_OK {
		return svtCDEFDecision{}, fmt.Errorf("%w: %s", errCUDASearch, C.GoString(C.pf_status_string(st)))
	}
	var p CDEFParams
	p.Damping = 3 + (qIndex >> 6)
	p.Bits = uint8(a.result.bits)
	for j := 0; j < int(a.result.strength_count) && j < MaxCDEFStrengths; j++ {
		p.YStrength[j] = uint8(a.result.y_strength[j])
		p.UVStrength[j] = uint8(a.result.uv_strength[j])
	}
	return svtCDEFDecision{params: p, fbIdx: s.fbIdx}, nil
}
