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
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
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

    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "kats.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote", dst)


if __name__ == "__main__":
    main()
