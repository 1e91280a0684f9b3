"""Generate pf_tables.h: the normative AV1 data tables the post-filter chain needs.

The tables are AV1 spec data (the 2048-entry film-grain Gaussian sequence,
the self-guided restoration tables and the super-resolution upscale filter).
They must match goav1 value for value, so they are parsed straight out of the
reference sources:

  internal/av1/filmgrain/gaussian.go        gaussianSequence
  internal/av1/restoration/selfguided.go    SGRParameterTable, xByXPlus1, oneByX
  internal/av1/superres/superres.go         upscaleFilter
  internal/av1/tile/partition.go            blockDimensions
  internal/av1/tile/tx_size.go              transformDimensions,
                                            maxTransformSizeForBlock

Run once where the reference checkout exists; the generated header is
committed, so builds elsewhere never read the reference.  The film-grain
table is checked against the checksums goav1's own test pins
(internal/av1/filmgrain/filmgrain_test.go:2129-2172) before anything is
written.

Usage: python goav1_b200/csrc/gen_tables.py /path/to/goav1
"""

import os
import re
import sys


def _block(text, start_pattern):
    m = re.search(start_pattern, text)
    if not m:
        raise SystemExit("pattern not found: " + start_pattern)
    depth = 0
    i = text.index("{", m.end() - 1)
    for j in range(i, len(text)):
        if text[j] == "{":
            depth += 1
        elif text[j] == "}":
            depth -= 1
            if depth == 0:
                return text[i + 1:j]
    raise SystemExit("unbalanced block after " + start_pattern)


def _ints(body):
    return [int(v) for v in re.findall(r"-?\d+", re.sub(r"//[^\n]*", "", body))]


def parse(ref):
    fg = open(os.path.join(ref, "internal/av1/filmgrain/gaussian.go")).read()
    gauss = _ints(_block(fg, r"var gaussianSequence = \[\.\.\.\]int16\{"))
    sg = open(os.path.join(ref, "internal/av1/restoration/selfguided.go")).read()
    params_body = _block(sg, r"var SGRParameterTable = \[SGRProjParams\]SGRParams\{")
    params = []
    for entry in re.findall(r"Radius: \[2\]uint8\{([^}]*)\}, S: \[2\]int16\{([^}]*)\}", params_body):
        r = [int(v) for v in entry[0].split(",")]
        s = [int(v) for v in entry[1].split(",")]
        params.append((r[0], r[1], s[0], s[1]))
    xby = _ints(_block(sg, r"var xByXPlus1 = \[256\]uint16\{"))
    oneby = _ints(_block(sg, r"var oneByX = \[25\]uint16\{"))
    sr = open(os.path.join(ref, "internal/av1/superres/superres.go")).read()
    upf = _ints(_block(sr, r"var upscaleFilter = \[FilterShifts\]\[FilterTaps\]int16\{"))
    tile = open(os.path.join(ref, "internal/av1/tile/partition.go")).read()
    bdim = re.findall(r"BlockSize(\d+)x(\d+):\s*\{W4: (\d+), H4: (\d+), Log2W: (\d+), Log2H: (\d+)\}",
                      _block(tile, r"var blockDimensions = \[blockSizeCount\]BlockDimensions\{"))
    txf = open(os.path.join(ref, "internal/av1/tile/tx_size.go")).read()
    consts = re.search(r"\tTransformSize4x4 TransformSize = iota\n(.*?)\ttransformSizeCount", txf, re.S).group(1)
    order = ["TransformSize4x4"] + re.findall(r"^\t(TransformSize\d+x\d+)$", consts, re.M)
    tdim = {}
    for m in re.finditer(r"(TransformSize\d+x\d+):\s*\{([^}]*)\}",
                         _block(txf, r"var transformDimensions = \[transformSizeCount\]TransformDimensions\{")):
        f = dict(kv.split(":") for kv in m.group(2).replace(" ", "").split(","))
        tdim[m.group(1)] = (int(f["W4"]), int(f["H4"]), int(f["Log2W"]), int(f["Log2H"]), f.get("Sub"))
    tx = []
    for name in order:
        w4, h4, lw, lh, sub = tdim[name]
        tx.append((w4, h4, lw, lh, order.index(sub) if sub else 0))
    maxtx = []
    for m in re.finditer(r"BlockSize(\d+)x(\d+):\s*\{([^}]*)\}",
                         _block(txf, r"var maxTransformSizeForBlock = \[blockSizeCount\]\[4\]TransformSize\{")):
        maxtx.append([order.index(v.strip()) for v in m.group(3).split(",")])
    blocks = [tuple(int(v) for v in b[2:]) + (int(b[0]), int(b[1])) for b in bdim]
    return gauss, params, xby, oneby, upf, blocks, tx, maxtx


def check(gauss, params, xby, oneby, upf, blocks, tx, maxtx):
    assert len(gauss) == 2048, len(gauss)
    s = sum(gauss)
    a = sum(abs(v) for v in gauss)
    w = sum((i + 1) * v for i, v in enumerate(gauss))
    if (s, a, w) != (1120, 837192, -8011268):
        raise SystemExit("gaussian checksum mismatch: %r" % ((s, a, w),))
    assert len(params) == 16 and len(xby) == 256 and len(oneby) == 25
    # 64 phases of 8 taps, each phase summing to 128 (unity gain).
    assert len(upf) == 64 * 8 and all(sum(upf[8 * i:8 * i + 8]) == 128 for i in range(64))
    # 22 block sizes and 19 transform sizes, each with its width and height in
    # 4x4 units consistent with its name and log2 classes.
    assert len(blocks) == 22 and len(tx) == 19 and len(maxtx) == 22
    for w4, h4, lw, lh, pw, ph in blocks:
        assert w4 * 4 == pw and h4 * 4 == ph and 1 << lw == w4 and 1 << lh == h4
    for i, (w4, h4, lw, lh, sub) in enumerate(tx):
        assert 1 << lw == w4 and 1 << lh == h4 and 0 <= sub < 19
        # A split quarters a square transform and halves a rectangular one.
        if i:
            assert tx[sub][0] * tx[sub][1] * (4 if w4 == h4 else 2) == w4 * h4
    assert all(len(r) == 4 and all(0 <= v < 19 for v in r) for r in maxtx)


def emit(gauss, params, xby, oneby, upf, blocks, tx, maxtx):
    out = []
    out.append("/* Generated by gen_tables.py from goav1's normative AV1 tables")
    out.append(" * (internal/av1/filmgrain/gaussian.go, internal/av1/restoration/selfguided.go,")
    out.append(" * internal/av1/superres/superres.go, internal/av1/tile/partition.go,")
    out.append(" * internal/av1/tile/tx_size.go).")
    out.append(" * Do not edit by hand. */")
    out.append("#ifndef PF_TABLES_H")
    out.append("#define PF_TABLES_H")
    out.append("#include <stdint.h>")
    out.append("")
    out.append("#define PF_GAUSSIAN_LEN 2048")
    out.append("static const int16_t pf_gaussian_sequence[PF_GAUSSIAN_LEN] = {")
    for i in range(0, len(gauss), 16):
        out.append("  " + ", ".join(str(v) for v in gauss[i:i + 16]) + ",")
    out.append("};")
    out.append("")
    out.append("/* {r0, r1, s0, s1} per SGR parameter set. */")
    out.append("static const int16_t pf_sgr_params[16][4] = {")
    for p in params:
        out.append("  {%d, %d, %d, %d}," % p)
    out.append("};")
    out.append("")
    out.append("static const uint16_t pf_sgr_x_by_xplus1[256] = {")
    for i in range(0, 256, 16):
        out.append("  " + ", ".join(str(v) for v in xby[i:i + 16]) + ",")
    out.append("};")
    out.append("")
    out.append("static const uint16_t pf_sgr_one_by_x[25] = {")
    out.append("  " + ", ".join(str(v) for v in oneby) + ",")
    out.append("};")
    out.append("")
    out.append("/* Super-resolution upscale filter: 64 subpel phases x 8 taps. */")
    out.append("static const int16_t pf_superres_filter[64][8] = {")
    for i in range(64):
        out.append("  {" + ", ".join(str(v) for v in upf[8 * i:8 * i + 8]) + "},")
    out.append("};")
    out.append("")
    out.append("/* Block sizes in goav1's tile.BlockSize order: {W4, H4} in 4x4 units. */")
    out.append("static const uint8_t pf_block_dims[22][2] = {")
    for b in blocks:
        out.append("  {%d, %d}," % b[:2])
    out.append("};")
    out.append("")
    out.append("/* Transform sizes in tile.TransformSize order: {W4, H4, Log2W, Log2H, Sub}. */")
    out.append("static const uint8_t pf_tx_dims[19][5] = {")
    for t in tx:
        out.append("  {%d, %d, %d, %d, %d}," % t)
    out.append("};")
    out.append("")
    out.append("/* Largest transform per block size: luma, 4:2:0, 4:2:2, 4:4:4 chroma. */")
    out.append("static const uint8_t pf_max_tx[22][4] = {")
    for r in maxtx:
        out.append("  {%d, %d, %d, %d}," % tuple(r))
    out.append("};")
    out.append("")
    out.append("#endif /* PF_TABLES_H */")
    return "\n".join(out) + "\n"


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GOAV1_REFERENCE")
    if not ref:
        sys.exit("usage: %s <path to a goav1 checkout> (or set GOAV1_REFERENCE)" % sys.argv[0])
    tabs = parse(ref)
    check(*tabs)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "pf_tables.h")
    with open(dst, "w") as f:
        f.write(emit(*tabs))
    print("wrote", dst)


if __name__ == "__main__":
    main()
