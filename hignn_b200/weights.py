"""Weight files for the learned two-body mobility kernel.

The reference ships its two-body network as a pickled ``torch.nn.Sequential``
(``nn/two_body_unbounded.pkl``: Linear(3,128) -> Tanh -> Linear(128,512) -> Tanh
-> Linear(512,9)) and converts it to a TorchScript ``.pt`` per device for
libtorch (python/convert.py:41-57, loaded at src/HignnModel.cpp:402-433).
This framework has no libtorch: the native library reads a flat
little-endian blob instead (extension ``.hgnw``):

    offset  type        meaning
    0       char[4]     magic "HGNW"
    4       u32         format version (1)
    8       u32         number of dense layers L
    12      u32         hidden activation (1 = tanh, 2 = SiLU)
    16      u32         output wrapper (1 = mobility: (y + I) / |r|, I for |r| < 1e-5;
                        2 = three-body: y / |r1| / |r2|; 3 = self: y / |r| / |r|)
    20      u32[2L]     (out_features, in_features) per layer
    ...     f32[]       per layer: weight (out x in, row-major), then bias (out)

The exporter needs torch only to unpickle the reference file; everything the
library reads at run time is this blob.
"""
from __future__ import annotations

import os
import struct
from dataclasses import dataclass

import numpy as np

MAGIC = b"HGNW"
VERSION = 1
ACT_TANH = 1
ACT_SILU = 2
WRAP_MOBILITY = 1
WRAP_THREE_BODY = 2
WRAP_SELF = 3


@dataclass
class MlpWeights:
    """Dense MLP weights as float32 numpy arrays (W: out x in, b: out)."""

    weights: list
    biases: list
    activation: int = ACT_TANH
    wrapper: int = WRAP_MOBILITY

    @property
    def dims(self):
        return [self.weights[0].shape[1]] + [w.shape[0] for w in self.weights]


def save_hgnw(path: str, mlp: MlpWeights) -> None:
    L = len(mlp.weights)
    with open(path, "wb") as fh:
        fh.write(MAGIC)
        fh.write(struct.pack("<4I", VERSION, L, mlp.activation, mlp.wrapper))
        for w in mlp.weights:
            fh.write(struct.pack("<2I", w.shape[0], w.shape[1]))
        for w, b in zip(mlp.weights, mlp.biases):
            fh.write(np.ascontiguousarray(w, dtype="<f4").tobytes())
            fh.write(np.ascontiguousarray(b, dtype="<f4").tobytes())


def load_hgnw(path: str) -> MlpWeights:
    with open(path, "rb") as fh:
        data = fh.read()
    if data[:4] != MAGIC:
        raise ValueError(f"{path}: not an HGNW weight file")
    version, L, act, wrap = struct.unpack_from("<4I", data, 4)
    if version != VERSION:
        raise ValueError(f"{path}: unsupported HGNW version {version}")
    off = 20
    shapes = []
    for _ in range(L):
        shapes.append(struct.unpack_from("<2I", data, off))
        off += 8
    ws, bs = [], []
    for o, i in shapes:
        w = np.frombuffer(data, dtype="<f4", count=o * i, offset=off).reshape(o, i).copy()
        off += 4 * o * i
        b = np.frombuffer(data, dtype="<f4", count=o, offset=off).copy()
        off += 4 * o
        ws.append(w)
        bs.append(b)
    if off != len(data):
        raise ValueError(f"{path}: trailing bytes in HGNW file")
    return MlpWeights(ws, bs, act, wrap)


def _load_reference_pickle(pkl_path: str, module_dir: str | None):
    """Unpickle a reference network. The three-body and self networks are pickled inside the
    wrappers of python/HIGNN/model_structure.py, which import torch_scatter at module level; a
    stand-in module is enough to unpickle them (scatter is not called)."""
    import sys
    import types

    import torch

    added = False
    if module_dir and module_dir not in sys.path:
        sys.path.insert(0, module_dir)
        added = True
    stub = "torch_scatter" not in sys.modules
    if stub:
        sys.modules["torch_scatter"] = types.SimpleNamespace(scatter=None)
    try:
        return torch.load(pkl_path, weights_only=False, map_location="cpu")
    finally:
        if stub:
            del sys.modules["torch_scatter"]
        if added:
            sys.path.remove(module_dir)


def export_pkl(pkl_path: str, out_path: str, wrapper: int = WRAP_MOBILITY, module_dir: str | None = None) -> MlpWeights:
    """Convert a reference ``nn.Sequential`` pickle (or a model_structure wrapper holding one as
    ``.net``) into an ``.hgnw`` blob."""
    import torch  # only needed to unpickle the reference file

    net = _load_reference_pickle(pkl_path, module_dir)
    if hasattr(net, "net") and isinstance(net.net, torch.nn.Module):
        net = net.net
    mods = list(net.children()) if hasattr(net, "children") else list(net)
    ws, bs, act = [], [], None
    for m in mods:
        if isinstance(m, torch.nn.Linear):
            ws.append(m.weight.detach().to(torch.float32).numpy().copy())
            bs.append(m.bias.detach().to(torch.float32).numpy().copy())
        elif isinstance(m, torch.nn.Tanh):
            act = ACT_TANH if act in (None, ACT_TANH) else None
        elif isinstance(m, torch.nn.SiLU):
            act = ACT_SILU if act in (None, ACT_SILU) else None
        else:
            raise ValueError(f"unsupported module in {pkl_path}: {m}")
    if act is None:
        raise ValueError(f"{pkl_path}: mixed or missing activations")
    mlp = MlpWeights(ws, bs, act, wrapper)
    save_hgnw(out_path, mlp)
    return mlp


def default_three_body_paths():
    """The shipped three-body and self networks (exported from the reference's
    python/Saved_Model/Unbounded/HIGNN_nn_{3body,self}.pkl)."""
    d = os.path.join(os.path.dirname(__file__), "data")
    return os.path.join(d, "three_body_unbounded.hgnw"), os.path.join(d, "self_unbounded.hgnw")


def default_two_body_path() -> str:
    """The shipped two-body weights (exported from nn/two_body_unbounded.pkl)."""
    return os.path.join(os.path.dirname(__file__), "data", "two_body_unbounded.hgnw")


def resolve_model_path(base: str) -> str:
    """Map the reference's base path (``<path>`` -> ``<path>_<dev>.pt``) to a blob.

    Accepts ``<path>.hgnw`` directly, ``<path>`` with a sibling ``.hgnw``, or a
    sibling ``.pkl`` that is exported next to it on first use.
    """
    if base.endswith(".hgnw") and os.path.exists(base):
        return base
    stem = base[:-4] if base.endswith(".pkl") else base
    cand = stem + ".hgnw"
    if os.path.exists(cand):
        return cand
    if os.path.exists(stem + ".pkl"):
        export_pkl(stem + ".pkl", cand)
        return cand
    raise FileNotFoundError(f"no two-body weights for '{base}' (looked for {cand}, {stem}.pkl)")


if __name__ == "__main__":
    import argparse

    ap = argparse.ArgumentParser(description="export a reference .pkl network to .hgnw")
    ap.add_argument("pkl")
    ap.add_argument("out")
    ap.add_argument("--wrapper", type=int, default=WRAP_MOBILITY,
                    help="1 two-body mobility, 2 three-body, 3 self")
    ap.add_argument("--module-dir", default=None,
                    help="directory holding the HIGNN package the pickle refers to (reference python/)")
    a = ap.parse_args()
    m = export_pkl(a.pkl, a.out, a.wrapper, a.module_dir)
    print("exported", a.out, "dims", m.dims)
