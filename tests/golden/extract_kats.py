"""Extract goav1's literal known-answer vectors for the post-filter path into kats.json.

Every vector below is copied by regex out of goav1's own Go test files, and
each entry records the file:line it came from.  The JSON is committed so the
tests never read the reference checkout at run time.

Usage: python tests/golden/extract_kats.py /path/to/goav1
"""

import json
import os
import re
import sys


def lineno(text, pos):
    return text.count("\n", 0, pos) + 1


def ints(s):
    return [int(v, 0) for v in re.findall(r"-?0x[0-9a-fA-F]+|-?\d+", s)]


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GOAV1_REFERENCE")
    if not ref:
        sys.exit("usage: %s <path to a goav1 checkout> (or set GOAV1_REFERENCE)" % sys.argv[0])
    out = {}

    p = "internal/av1/filmgrain/filmgrain_test.go"
    t = open(os.path.join(ref, p)).read()
    m = re.search(r"func TestRandomNumber\(t \*testing.T\) \{.*?NewRandom\((0x[0-9a-f]+)\).*?wantValues := \[\]uint16\{([^}]*)\}.*?wantRegisters := \[\]uint16\{([^}]*)\}", t, re.S)
    out["lfsr8"] = {"src": "%s:%d" % (p, lineno(t, m.start())), "seed": int(m.group(1), 16),
                    "values": ints(m.group(2)), "registers": ints(m.group(3))}
    m = re.search(r"func TestRandomNumberElevenBits.*?NewRandom\((0x[0-9a-f]+)\).*?range \[\]uint16\{([^}]*)\}", t, re.S)
    out["lfsr11"] = {"src": "%s:%d" % (p, lineno(t, m.start())), "seed": int(m.group(1), 16), "values": ints(m.group(2))}
    m = re.search(r"func TestRandomSeeds.*?NewPlaneRandom\((0x[0-9a-f]+), 1\).*?cb.register != (0x[0-9a-f]+).*?cr.register != (0x[0-9a-f]+).*?NewStripeRandom\((0x[0-9a-f]+), (\d+)\).*?stripe.register != (0x[0-9a-f]+)", t, re.S)
    out["fg_seeds"] = {"src": "%s:%d" % (p, lineno(t, m.start())), "seed": int(m.group(1), 16),
                       "cb": int(m.group(2), 16), "cr": int(m.group(3), 16),
                       "stripe_line": int(m.group(5)), "stripe": int(m.group(6), 16)}
    m = re.search(r"func TestGaussianSequence\(t.*?sum != (-?\d+) \|\| abs != (-?\d+) \|\| weighted != (-?\d+).*?wantFirst := \[\.\.\.\]int16\{([^}]*)\}.*?wantMid := \[\.\.\.\]int16\{([^}]*)\}.*?index := (\d+) \+ i.*?wantLast := \[\.\.\.\]int16\{([^}]*)\}", t, re.S)
    out["gaussian"] = {"src": "%s:%d" % (p, lineno(t, m.start())), "sum": int(m.group(1)), "abs": int(m.group(2)),
                       "weighted": int(m.group(3)), "first": ints(m.group(4)), "mid_start": int(m.group(6)),
                       "mid": ints(m.group(5)), "last": ints(m.group(7))}
    m = re.search(r"func TestBuildScalingLUT\(t \*testing.T\) \{(.*?)\n\t\}\n\tfor", t, re.S)
    cases = []
    for c in re.finditer(r"name:\s*\"([^\"]+)\",(.*?)samples: map\[int\]uint8\{([^}]*)\}", m.group(1), re.S):
        pts = [[int(a), int(b)] for a, b in re.findall(r"Value: (\d+), Scaling: (\d+)", c.group(2))]
        samples = {int(k): int(v) for k, v in re.findall(r"(\d+): (\d+)", c.group(3))}
        cases.append({"name": c.group(1), "points": pts, "samples": samples})
    out["scaling_lut"] = {"src": "%s:%d" % (p, lineno(t, m.start())), "cases": cases}

    p = "internal/av1/cdef/cdef_test.go"
    t = open(os.path.join(ref, p)).read()
    m = re.search(r"func TestFindDirectionKnownPatterns", t)
    body = t[m.start():m.start() + 2000]
    dirs = [(n, int(d), int(v)) for n, d, v in re.findall(r"name: \"(\w+)\",.*?wantDir: (\d+),\s*wantVar: (\d+)", body, re.S)]
    out["cdef_dir"] = {"src": "%s:%d" % (p, lineno(t, m.start())),
                       "cases": [{"name": n, "dir": d, "var": v} for n, d, v in dirs]}

    p = "internal/av1/loopfilter/loopfilter_test.go"
    t = open(os.path.join(ref, p)).read()
    m = re.search(r"func TestFilter14EdgeQ32Row7", t)
    body = t[m.start():m.start() + 6000]
    rows = [ints(r) for r in re.findall(r"/\* y=\s*\d+\s*\*/ \{([^}]*)\}", body)]
    lvl = re.search(r"ThresholdsForLevel\((\d+), (\d+)\)", body)
    out["filter14_q32_row7"] = {"src": "%s:%d" % (p, lineno(t, m.start())), "rows": rows, "bit_depth": 10,
                                "level": int(lvl.group(1)), "sharpness": int(lvl.group(2)), "edge_x": 16,
                                "unchanged": [[16, 7]]}

    p = "internal/av1/restoration/restoration_test.go"
    t = open(os.path.join(ref, p)).read()
    m = re.search(r"func TestDecodeSGRXQMatchesLibaom.*?\n\}", t, re.S)
    cases = [{"set": int(s), "xqd": ints(x), "want": ints(w)} for s, x, w in re.findall(
        r"SGRParameterTable\[(\d+)\], xqd: \[2\]int8\{([^}]*)\}, want: \[2\]int16\{([^}]*)\}", m.group(0))]
    out["sgr_xq"] = {"src": "%s:%d" % (p, lineno(t, m.start())), "cases": cases}
    m = re.search(r"xByXPlus1Checks := map\[uint32\]int32\{([^}]*)\}", t)
    out["sgr_x_by_xplus1"] = {"src": "%s:%d" % (p, lineno(t, m.start())),
                              "checks": {int(k): int(v) for k, v in re.findall(r"(\d+):\s*(\d+)", m.group(1))}}
    m = re.search(r"func TestDefaultWienerInfoMatchesLibaom.*?want := WienerFilter\{([^}]*)\}.*?roundTests := map\[uint8\]\[2\]int\{(.*?)\n\t\}", t, re.S)
    out["wiener"] = {"src": "%s:%d" % (p, lineno(t, m.start())), "default": ints(m.group(1)),
                     "rounds": {int(k): ints(v) for k, v in re.findall(r"(\d+):\s*\{([^}]*)\}", m.group(2))}}

    p = "internal/av1/superres/superres_test.go"
    t = open(os.path.join(ref, p)).read()
    m = re.search(r"func TestUpscalePlaneMatchesNormativeRows", t)
    cases = [{"name": n, "bit_depth": int(b), "src": ints(s_), "dst_width": int(w), "want": ints(wa)}
             for n, b, s_, w, wa in re.findall(
                 r"name:\s*\"([^\"]+)\",\s*bitDepth: (\d+),\s*src:\s*\[\]uint16\{([^}]*)\},\s*dstWidth: (\d+),"
                 r"\s*want:\s*\[\]uint16\{([^}]*)\}", t[m.start():], re.S)]
    out["superres_rows"] = {"src": "%s:%d" % (p, lineno(t, m.start())), "cases": cases}
    p = "internal/av1/superres/superres_aligned_libaom_test.go"
    t = open(os.path.join(ref, p)).read()
    m = re.search(r"func TestUpscalePlaneCodedMatchesLibaomAlignedRow.*?src := \[\]uint16\{([^}]*)\}.*?want := "
                  r"\[\]uint16\{([^}]*)\}.*?codedWidth = (\d+).*?alignedWidth = (\d+).*?upscaledWidth = (\d+)", t, re.S)
    out["superres_libaom_row"] = {"src": "%s:%d" % (p, lineno(t, m.start())), "src_row": ints(m.group(1)),
                                  "want": ints(m.group(2)), "coded_width": int(m.group(3)),
                                  "aligned_width": int(m.group(4)), "upscaled_width": int(m.group(5)), "bit_depth": 8}


    # Deblocking edge filters with explicit thresholds: every literal
    # Filter4/6/8/14Edge known-answer test (one sample line across the edge,
    # the same on every line along it) and the sample lists the
    # MatchesCReference tests feed to goav1's libaom restatement.
    p = "internal/av1/loopfilter/loopfilter_test.go"
    t = open(os.path.join(ref, p)).read()
    edge_kats = []
    for m in re.finditer(r"func (TestFilter(4|6|8|14)Edge(\w+))\(t \*testing.T\) \{(.*?)\n\}\n", t, re.S):
        name, width, body = m.group(1), int(m.group(2)), m.group(4)
        if any(k in name for k in ("MatchesCReference", "Rejects", "Allocs", "Q32Row7")):
            continue
        call = re.search(r"Filter\d+Edge\(plane, (\d), (\w+), Edge(Horizontal|Vertical), (\d+), (\d+), (\d+), "
                         r"(thresholds|Thresholds\{[^}]*\})", body)
        if not call:
            continue
        thr_src = call.group(7)
        if thr_src == "thresholds":
            thr_src = re.search(r"thresholds := Thresholds\{([^}]*)\}", body).group(1)
        thr = {k: int(v) for k, v in re.findall(r"(\w+): (\d+)", thr_src)}
        horizontal = call.group(3) == "Horizontal"
        q0 = int(call.group(5)) if horizontal else int(call.group(4))
        depths = [int(call.group(2))] if call.group(2).isdigit() else \
            ints(re.search(r"range \[\]uint8\{([^}]*)\}", body).group(1))
        line = {}
        for c in re.finditer(r"setSample\(plane, \d, (\w+), (\w+), (\d+)\)", body):
            a, b, v = c.group(1), c.group(2), int(c.group(3))
            pos = b if horizontal else a
            if pos.isdigit():
                line[int(pos)] = v
        # Loops over the coordinate across the edge (the filter14 tests).
        for c in re.finditer(r"for (\w+) := range (\d+) \{\s*setSample\(plane, \d, (\w+), (\w+), (\d+)\)", body):
            if c.group(1) == (c.group(4) if horizontal else c.group(3)):
                for k in range(int(c.group(2))):
                    line[k] = int(c.group(5))
        for c in re.finditer(r"for (\w+) := (\d+); \w+ < (\d+); \w+\+\+ \{\s*setSample\(plane, \d, (\w+), (\w+), "
                             r"(\d+)\)", body):
            if c.group(1) == (c.group(5) if horizontal else c.group(4)):
                for k in range(int(c.group(2)), int(c.group(3))):
                    line[k] = int(c.group(6))
        want = {}
        for c in re.finditer(r"getSample\(plane, \d, (\w+), (\w+)\); got != (\d+)", body):
            pos = c.group(2) if horizontal else c.group(1)
            if pos.isdigit():
                want[int(pos)] = int(c.group(3))
        w = re.search(r"want := \[\]uint16\{([^}]*)\}", body)
        if w:
            want = dict(enumerate(ints(w.group(1))))
        edge_kats.append({"name": name, "src": "%s:%d" % (p, lineno(t, m.start())), "width": width,
                          "bit_depths": depths, "limit": thr.get("Limit", 0), "blimit": thr.get("BlockLimit", 0),
                          "hev": thr.get("HighEdgeVariance", 0), "q0": q0,
                          "line": [line[k] for k in sorted(line)], "want": {str(k): v for k, v in want.items()}})
    out["lf_edge_kats"] = edge_kats
    cref = []
    for m in re.finditer(r"func (TestFilter(4|6|8|14)EdgeMatchesCReference)\(t \*testing.T\) \{(.*?)\n\}\n", t, re.S):
        for c in re.finditer(r"bitDepth:\s*(\d+),\s*thresholds: Thresholds\{([^}]*)\},\s*samples: \[\]\[\d+\]int\{(.*?)\n\t\t\t\},",
                             m.group(3), re.S):
            thr = {k: int(v) for k, v in re.findall(r"(\w+): (\d+)", c.group(2))}
            cref.append({"src": "%s:%d" % (p, lineno(t, m.start())), "width": int(m.group(2)),
                         "bit_depth": int(c.group(1)), "limit": thr.get("Limit", 0),
                         "blimit": thr.get("BlockLimit", 0), "hev": thr.get("HighEdgeVariance", 0),
                         "samples": [ints(r) for r in re.findall(r"\{([^{}]*)\}", c.group(3))]})
    out["lf_cref_samples"] = cref
    m = re.search(r"func TestThresholdsForLevel\(t \*testing.T\) \{(.*?)\n\}\n", t, re.S)
    out["lf_thresholds"] = {"src": "%s:%d" % (p, lineno(t, m.start())), "cases": [
        {"level": int(a), "sharpness": int(b), "limit": int(c), "blimit": int(d), "hev": int(e)}
        for a, b, c, d, e in re.findall(r"level: (\d+), sharpness: (\d+), want: Thresholds\{Limit: (\d+), "
                                        r"BlockLimit: (\d+), HighEdgeVariance: (\d+)\}", m.group(1))]}

    # CDEF: the chroma direction conversion of a 4:2:2 plane.
    p = "internal/av1/cdef/cdef_test.go"
    t = open(os.path.join(ref, p)).read()
    m = re.search(r"func TestFilterFrameBlocksConvertsChromaDirections.*?XDec:\s*(\d+),.*?want := \[\]uint8\{([^}]*)\}",
                  t, re.S)
    out["cdef_chroma_dir"] = {"src": "%s:%d" % (p, lineno(t, m.start())), "xdec": int(m.group(1)), "ydec": 0,
                              "luma_dirs": list(range(len(ints(m.group(2))))), "want": ints(m.group(2))}

    # Loop restoration: the SGR parameter table (radius and s per pass).
    p = "internal/av1/restoration/restoration_test.go"
    t = open(os.path.join(ref, p)).read()
    m = re.search(r"func TestSGRParameterTableMatchesLibaom.*?want := \[SGRProjParams\]SGRParams\{(.*?)\n\t\}", t, re.S)
    out["sgr_params"] = {"src": "%s:%d" % (p, lineno(t, m.start())), "sets": [
        {"radius": ints(r), "s": ints(s_)} for r, s_ in
        re.findall(r"Radius: \[2\]uint8\{([^}]*)\}, S: \[2\]int16\{([^}]*)\}", m.group(1))]}
    m = re.search(r"oneByX\[0\] != (\d+) \|\| oneByX\[24\] != (\d+)", t)
    out["sgr_one_by_x"] = {"src": "%s:%d" % (p, lineno(t, m.start())), "n1": int(m.group(1)), "n25": int(m.group(2))}

    # Film grain: the literal ApplyLumaRow / ApplyChromaRow tests (one
    # 32-row stripe band with templates set at the offsets the stripe's
    # LFSR draws, checked samples).
    p = "internal/av1/filmgrain/filmgrain_test.go"
    t = open(os.path.join(ref, p)).read()
    consts = {}
    for f in ("constants.go", "blend.go"):
        consts.update({k: int(v) for k, v in re.findall(r"^\t(\w+)\s*=\s*(\d+)$", open(os.path.join(
            ref, "internal/av1/filmgrain", f)).read(), re.M)})
    rows = []
    for m in re.finditer(r"func (TestApply(Luma|Chroma)Row(NoOverlap|LeftOverlap|TopOverlap|CornerOverlap|"
                         r"UsesChromaScalingFormula|LeftOverlap420|TopOverlap420|CornerOverlap420|ClipsRestrictedRange))"
                         r"\(t \*testing.T\) \{(.*?)\n\}\n", t, re.S):
        name, kind, body = m.group(1), m.group(2).lower(), m.group(4)
        dims = {k: int(v) for k, v in re.findall(r"(width|height|stride|lumaStride)\s*=\s*(\d+)", body)}
        src_val = int(re.search(r"test\w+RowBuffers\(width, height, stride, (\d+)\)", body).group(1))
        lm = re.search(r"testChromaRowLuma\([^)]*, (\d+)\)", body)
        lut = {"fill": 0, "set": {}}
        lf = re.search(r"testLumaRowScaling\((\d+)\)", body)
        if lf:
            lut["fill"] = int(lf.group(1))
        for k, v in re.findall(r"lut\[(\d+)\] = (\d+)", body):
            lut["set"][k] = int(v)
        sets = []
        for c in re.finditer(r"setTest(Luma|Chroma)RowGrain\(t, grain, (0x[0-9a-f]+), (.*?)\)\n", body):
            f = [x.strip() for x in c.group(3).split(",")]
            if c.group(1) == "Chroma":
                f = f[2:]  # the subsampling flags repeat the params
            sets.append({"offset": int(c.group(2), 16), "block_col": int(f[0]), "block_row": int(f[1]),
                         "x": int(f[2]), "y": int(f[3]), "value": int(f[4])})
        pm = re.search(r"params := \w+RowParams\{(.*?)\n\t\}", body, re.S).group(1)
        params = {}
        for k, v in re.findall(r"(\w+):\s*(\w+),", pm):
            params[k] = {"true": 1, "false": 0}.get(v, dims.get(v, int(v) if v.isdigit() else v))
        checks = []
        for c in re.finditer(r"dst\[(\w+)\]; got != (\w+)", body):
            idx, val = c.group(1), c.group(2)
            idx = dims.get(idx, int(idx) if idx.isdigit() else idx)
            val = int(val) if val.isdigit() else consts[val]
            checks.append({"index": idx, "want": val})
        rows.append({"name": name, "src": "%s:%d" % (p, lineno(t, m.start())), "plane": kind, "dims": dims,
                     "src_value": src_val, "luma_value": int(lm.group(1)) if lm else None, "lut": lut,
                     "grain": sets, "params": params, "checks": checks})
    out["fg_rows"] = rows

    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "kats.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote", dst)


if __name__ == "__main__":
    main()
