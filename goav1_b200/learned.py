"""Learned CDEF strength selection: model files, labels, datasets, training.

The network and its kernels live in the library (pf_mlp.cu, entry points
pf_cdef_features / pf_cdef_mlp_* / pf_cdef_search_learned); this module is
the host-side glue a user needs to build a model:

* ``init_model`` - He-initialised weights (rounded to bf16) and the feature
  normalisation taken from the training features.
* ``canonical_labels`` - per filter block, the trial index the network learns
  for each head, from the exhaustive search's SSE table.  Trials within
  ``tie`` (relative) of the block's minimum are near-ties; among them the
  label is the one the frame as a whole prefers (lowest total SSE over the
  frame's blocks), which gives the network one consistent answer for
  interchangeable trials and keeps the labels of one frame pointing at the
  strengths its preset selection will pick.  (Ranking near-ties by a global
  prior instead drags every block of a frame towards the same off-frame
  choice; within the tolerance per block, the frame loses up to the whole
  tolerance.)
* ``make_dataset`` - features and labels of seeded synthetic frames: source
  without noise, reconstruction with per-8x8 DC offsets and Gaussian noise,
  deblocked by the library, searched exhaustively by the library.
* ``python -m goav1_b200.learned train`` - builds the dataset, trains on the
  GPU and writes the model file.

The model file is the raw ``pf_cdef_mlp`` struct preceded by an 8-byte magic.
"""

import argparse
import ctypes as C
import json
import os
import time

import numpy as np

from . import abi, synth

MAGIC = b"PFMLP01\0"
DEFAULT_MODEL = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "cdef_mlp_1080p.bin")
QINDEX_CHOICES = (64, 96, 128, 160, 192)
LAMBDA = 4000.0


def bf16_bits(x):
    """float32 array -> bf16 bit patterns (round to nearest, ties to even)."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return r.astype(np.uint16)


def bf16_float(b):
    return (np.asarray(b, np.uint16).astype(np.uint32) << 16).view(np.float32)


def model_arrays(m):
    """Copies of a pf_cdef_mlp's parameters as float32 numpy arrays."""
    return {
        "w1": bf16_float(np.ctypeslib.as_array(m.w1)).reshape(abi.PF_MLP_HIDDEN, abi.PF_MLP_FEATURES),
        "w2": bf16_float(np.ctypeslib.as_array(m.w2)).reshape(abi.PF_MLP_HIDDEN, abi.PF_MLP_HIDDEN),
        "w3": bf16_float(np.ctypeslib.as_array(m.w3)).reshape(abi.PF_MLP_OUTPUTS, abi.PF_MLP_HIDDEN),
        "b1": np.ctypeslib.as_array(m.b1).copy(),
        "b2": np.ctypeslib.as_array(m.b2).copy(),
        "b3": np.ctypeslib.as_array(m.b3).copy(),
        "shift": np.ctypeslib.as_array(m.feat_shift).copy(),
        "scale": np.ctypeslib.as_array(m.feat_scale).copy(),
    }


def init_model(X, seed=0):
    """A fresh model: He-normal weights rounded to bf16, zero biases, and
    (x - mean) / std feature normalisation from the training features X."""
    rng = np.random.default_rng([seed, 0xC0DE])
    m = abi.pf_cdef_mlp()
    F, H, O = abi.PF_MLP_FEATURES, abi.PF_MLP_HIDDEN, abi.PF_MLP_OUTPUTS
    for name, fan_in, shape in (("w1", F, (H, F)), ("w2", H, (H, H)), ("w3", H, (O, H))):
        w = rng.standard_normal(shape).astype(np.float32) * np.float32(np.sqrt(2.0 / fan_in))
        np.ctypeslib.as_array(getattr(m, name))[:] = bf16_bits(w).ravel()
    mean = X.mean(0).astype(np.float32)
    std = X.std(0).astype(np.float32)
    np.ctypeslib.as_array(m.feat_shift)[:] = mean
    np.ctypeslib.as_array(m.feat_scale)[:] = np.where(std > 1e-6, 1.0 / np.maximum(std, 1e-6), 0.0).astype(np.float32)
    return m


def save_model(m, path):
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "wb") as f:
        f.write(MAGIC)
        f.write(bytes(m))


def load_model(path=DEFAULT_MODEL):
    with open(path, "rb") as f:
        data = f.read()
    if data[:8] != MAGIC or len(data) != 8 + C.sizeof(abi.pf_cdef_mlp):
        raise ValueError("%s is not a pf_cdef_mlp model file" % path)
    return abi.pf_cdef_mlp.from_buffer_copy(data[8:])


def argmin_prior(tables):
    """Trial preference order per head: trials sorted by how often they are
    the exhaustive argmin over the given (mse, keep) tables, most often first
    (ties to the lower index)."""
    counts = np.zeros((2, 64), np.int64)
    for mse, keep in tables:
        for p in range(2):
            counts[p] += np.bincount(mse[p][keep].argmin(1), minlength=64)
    return np.stack([np.lexsort((np.arange(64), -counts[p])) for p in range(2)])


def frame_prior(mse, keep):
    """Per head, the trials of one frame ordered by their total SSE over the
    frame's searched blocks (ties to the lower index)."""
    return np.stack([np.lexsort((np.arange(64), mse[p][keep].astype(np.float64).sum(0))) for p in range(2)])


def canonical_labels(mse, keep, prior=None, tie=0.01):
    """Labels (n, 2) uint8 for the filter blocks `keep` of one SSE table;
    near-ties ranked by `prior` (default: the frame's own ranking)."""
    if prior is None:
        prior = frame_prior(mse, keep)
    out = np.zeros((int(keep.sum()), 2), np.uint8)
    for p in range(2):
        m = mse[p][keep].astype(np.float64)
        best = m.min(1, keepdims=True)
        near = m <= best * (1.0 + tie)
        rank = np.empty(64, np.int64)
        rank[prior[p]] = np.arange(64)
        score = np.where(near, rank[None, :], 1 << 20)
        out[:, p] = score.argmin(1)
    return out


def strength_trial(packed):
    """Packed CDEF strength -> its index in the level-1 trial order."""
    return packed // 4 if packed % 4 == 0 else 16 + (packed // 4) * 3 + (packed % 4) - 1


def luma_sse(res, idx, mse_exh):
    """Luma SSE over the searched blocks under a decision (presets `res`,
    per-block index `idx`), read from an exhaustive table: the table holds
    the SSE of every trial of every block, so this is the SSE the decision
    gives without filtering the frame again."""
    live = np.nonzero(mse_exh[0].sum(1) > 0)[0]
    return int(sum(int(mse_exh[0][fb][strength_trial(res.y_strength[idx[fb]])]) for fb in live))


def frame_qindex(seed):
    return int(np.random.default_rng([seed, 0x9D]).choice(QINDEX_CHOICES))


def noskip_of(side, fr):
    ucols, urows = (fr.width + 63) // 64, (fr.height + 63) // 64
    return np.ctypeslib.as_array((C.c_uint8 * (ucols * urows * 8)).from_address(side.side.cdef.noskip)).copy()


def _gen(args):
    seed, w, h = args
    src, rec, side, sigma = synth.make_search_pair(seed, w, h)
    return seed, src, rec, side, sigma


def search_frames(seeds, width, height, workers=8):
    """Yields (seed, src, rec, side, sigma) for each seed; frames are made by
    a spawn-started process pool (no CUDA in the workers)."""
    if workers <= 1:
        for s in seeds:
            yield _gen((s, width, height))
        return
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    with ctx.Pool(workers) as pool:
        for item in pool.imap(_gen, [(s, width, height) for s in seeds]):
            yield item


def make_dataset(runner, seeds, width=1920, height=1080, workers=8):
    """(X float32[n, 40], tables) over the given seeds: the deblocked
    reconstruction's features and the exhaustive SSE table of each frame.
    tables: list of (seed, mse, keep, qindex)."""
    Xs, tables = [], []
    for seed, src, rec, side, sigma in search_frames(seeds, width, height, workers):
        runner.apply(rec.pf(), side.side)  # deblock (the side info's stages are loop filter only)
        ns = noskip_of(side, rec)
        q = frame_qindex(seed)
        _, mse, _ = runner.cdef_search(src.pf(), rec.pf(), ns, q, LAMBDA)
        X = runner.cdef_features(rec.pf(), ns, q)
        keep = mse[0].sum(1) > 0
        Xs.append(X[keep])
        tables.append((seed, mse, keep, q))
    return np.concatenate(Xs), tables


def parse_seeds(text):
    a, b = text.split("-")
    return list(range(int(a), int(b) + 1))


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m goav1_b200.learned")
    sub = ap.add_subparsers(dest="cmd", required=True)
    tr = sub.add_parser("train", help="generate the dataset, train on the GPU, write the model")
    tr.add_argument("--seeds", default="1000-1199")
    tr.add_argument("--size", default="1920x1080")
    tr.add_argument("--epochs", type=int, default=40)
    tr.add_argument("--batch", type=int, default=256)
    tr.add_argument("--lr", type=float, default=2e-3)
    tr.add_argument("--tie", type=float, default=0.01)
    tr.add_argument("--workers", type=int, default=8)
    tr.add_argument("--out", default=DEFAULT_MODEL)
    args = ap.parse_args(argv)
    from .postfilter import PostFilterRunner

    w, h = (int(v) for v in args.size.split("x"))
    runner = PostFilterRunner()
    t0 = time.time()
    X, tables = make_dataset(runner, parse_seeds(args.seeds), w, h, args.workers)
    t1 = time.time()
    prior = argmin_prior([(m, k) for _, m, k, _ in tables])  # reported: the no-network baseline uses it
    Y = np.concatenate([canonical_labels(m, k, None, args.tie) for _, m, k, _ in tables])
    model = init_model(X, seed=1)
    losses = runner.mlp_train(model, X, Y, args.epochs, batch=args.batch, lr=args.lr)
    t2 = time.time()
    P = runner.mlp_forward(model, X)
    acc = [(P[:, 64 * p:64 * (p + 1)].argmax(1) == Y[:, p]).mean() for p in range(2)]
    conf = ((P[:, :64].max(1) >= 0.5) & (P[:, 64:].max(1) >= 0.5)).mean()
    save_model(model, args.out)
    report = {"command": "python -m goav1_b200.learned train --seeds %s --size %s --epochs %d --batch %d --lr %g "
                         "--tie %g" % (args.seeds, args.size, args.epochs, args.batch, args.lr, args.tie),
              "samples": int(X.shape[0]), "loss_first": float(losses[0]), "loss_last": float(losses[-1]),
              "train_top1_acc_luma": float(acc[0]), "train_top1_acc_chroma": float(acc[1]),
              "train_confident_frac": float(conf),
              "prior_luma": prior[0][:8].tolist(), "prior_chroma": prior[1][:8].tolist(),
              "dataset_s": round(t1 - t0, 1), "train_s": round(t2 - t1, 2)}
    with open(os.path.splitext(args.out)[0] + ".json", "w") as f:
        json.dump(report, f, indent=1)
    print(json.dumps(report))
    runner.close()


if __name__ == "__main__":
    main()
