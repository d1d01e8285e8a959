"""StereoNet checkpoints: the reference's plain-text format and a packed copy.

The text format is the one ``save_weights`` writes (stereonet.py:1766-1787):
a header line ``stereonet feat_C=.. cost_C=.. D=.. max_disp=.. refine_C=..
refine_dil=a,b,c target_peak=..``, the block count, then one line per
parameter block ``n v1 .. vn`` in ``StereoNet.all_params()`` order
(stereonet.py:1193-1195).  Headerless files written before the header existed
are matched against the architectures the reference shipped, as
``load_model`` does (stereonet.py:1826-1853).

The packed copy (``weights/stereonet_weights.npz``) holds the same FP64
values, parsed with Python's ``float`` exactly as ``load_weights`` does
(stereonet.py:1856-1874), so the GPU box needs no text parsing.
"""

from __future__ import annotations

import dataclasses
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_NPZ = os.path.join(_HERE, "weights", "stereonet_weights.npz")


@dataclasses.dataclass
class NetArch:
    feat_C: int = 8
    cost_C: int = 4
    D: int = 8
    max_disp: int = 32
    refine_C: int = 8
    refine_dil: tuple = (1, 2, 4)
    target_peak: int = 20

    def block_sizes(self):
        C, Cm, Rc = self.feat_C, self.cost_C, self.refine_C
        s = []
        for ic in (1, C, C, C):                       # FeatureNet c1..c4, 3x3
            s += [C * ic * 9, C]
        for ic, oc in ((C, Cm), (Cm, Cm), (Cm, 1)):   # CostFilter, 3x3x3
            s += [oc * ic * 27, oc]
        for _ in range(2):                            # Refinement x2
            prev = 2
            for _d in self.refine_dil:
                s += [Rc * prev * 9, Rc]
                prev = Rc
            s += [prev * 9, 1]
        return s

    def vector(self):
        """arch ints as the C ABI takes them: C, Cm, D, Rc, ndil, dil..."""
        return [self.feat_C, self.cost_C, self.D, self.refine_C,
                len(self.refine_dil)] + list(self.refine_dil)


@dataclasses.dataclass
class StereoNetWeights:
    arch: NetArch
    blocks: list          # list of float64 arrays, all_params() order

    @property
    def flat(self) -> np.ndarray:
        return np.concatenate(self.blocks).astype(np.float64)

    @property
    def target_peak(self) -> float:
        return float(self.arch.target_peak)

    def n_params(self) -> int:
        return int(sum(len(b) for b in self.blocks))


_LEGACY = [(8, 4, 4, (1, 2)), (8, 4, 8, (1, 2, 4)), (12, 6, 8, (1, 2, 4)),
           (16, 8, 8, (1, 2, 4))]


def _parse_header(line: str) -> NetArch | None:
    if not line.startswith("stereonet "):
        return None
    a = NetArch()
    for tok in line.split()[1:]:
        if "=" not in tok:
            continue
        k, v = tok.split("=", 1)
        if k == "refine_dil":
            a.refine_dil = tuple(int(d) for d in v.split(","))
        elif hasattr(a, k):
            setattr(a, k, int(v))
    return a


def load_text(path: str) -> StereoNetWeights:
    """Parse a reference text checkpoint (``load_model`` semantics)."""
    with open(path) as f:
        lines = f.read().split("\n")
    arch = _parse_header(lines[0].strip())
    off = 1 if arch is not None else 0
    count = int(lines[off])
    blocks = []
    for k in range(count):
        parts = lines[k + 1 + off].split()
        n = int(parts[0])
        blocks.append(np.array([float(v) for v in parts[1:n + 1]], dtype=np.float64))
    sizes = [len(b) for b in blocks]
    if arch is None:
        for fc, cc, rc, dil in _LEGACY:
            cand = NetArch(fc, cc, 8, 32, rc, dil, 20)
            if cand.block_sizes() == sizes:
                arch = cand
                break
        else:
            raise ValueError("checkpoint %s does not match any known architecture" % path)
    if arch.block_sizes() != sizes:
        raise ValueError("checkpoint does not match model")
    return StereoNetWeights(arch, blocks)


def save_npz(w: StereoNetWeights, path: str) -> None:
    a = w.arch
    np.savez(path, arch=np.array([a.feat_C, a.cost_C, a.D, a.max_disp, a.refine_C,
                                  a.target_peak] + list(a.refine_dil), dtype=np.int64),
             **{"block_%02d" % i: b for i, b in enumerate(w.blocks)})


def load_npz(path: str = DEFAULT_NPZ) -> StereoNetWeights:
    z = np.load(path)
    v = [int(t) for t in z["arch"]]
    arch = NetArch(v[0], v[1], v[2], v[3], v[4], tuple(v[6:]), v[5])
    n = len([k for k in z.files if k.startswith("block_")])
    blocks = [z["block_%02d" % i].astype(np.float64) for i in range(n)]
    if arch.block_sizes() != [len(b) for b in blocks]:
        raise ValueError("packed checkpoint does not match its architecture")
    return StereoNetWeights(arch, blocks)


def load_model(path: str | None = None) -> StereoNetWeights:
    """Weights from a text checkpoint or a packed ``.npz`` (default: the
    packed copy of the reference's ``stereonet_weights.txt``)."""
    if path is None:
        return load_npz(DEFAULT_NPZ)
    if path.endswith(".npz"):
        return load_npz(path)
    return load_text(path)


if __name__ == "__main__":
    import sys
    if len(sys.argv) != 3:
        print("usage: python weights.py <stereonet_weights.txt> <out.npz>")
        sys.exit(2)
    w = load_text(sys.argv[1])
    save_npz(w, sys.argv[2])
    print("packed %d blocks, %d params, arch %s" % (len(w.blocks), w.n_params(), w.arch))
