"""B200-native (sm_100a) disparity hot path of Ray-5106/From-Scratch-Stereo-Vision.

The package directory name is not a Python identifier; load it through
``__graft_entry__.load_package()`` (which registers it as ``sv_b200``) or
with ``importlib`` the same way.  Modules:

* ``refine``  -- census / band_costs / _aggregate_path / refine_fullres /
  left_to_right / lr_refine drop-ins (stereonet.py:5115-5391);
* ``network`` -- StereoNet.forward, predict, predict_at_scale, predict_auto
  drop-ins (stereonet.py:998-1268, 3832-3961, 5891-5897);
* ``pipeline``-- the network + refinement path for one pair, device resident;
* ``shim``    -- ``install(SN)`` rebinds those names in an exec'd reference
  namespace, so the reference's own callers use the GPU versions;
* ``post``    -- median_filter / slic / plane_snap / refine_disparity /
  lr_consistency / fill_invalid drop-ins; ``band`` -- the learned band;
* ``image``   -- read_png / read_pnm / read_image drop-ins (host decode,
  GPU FP64 conversion);
* ``train``   -- StereoNet training (train_grads / train_step drop-ins and a
  device-resident batched ``Trainer``);
* ``synth``   -- seeded synthetic stereo pairs; ``weights`` -- checkpoints.

All compute goes through libsv_b200.so; there is no CPU fallback.
"""

from . import _lib, synth, weights  # noqa: F401

__all__ = ["_lib", "synth", "weights"]


def __getattr__(name):
    # heavy modules (torch) load on first use
    import importlib
    if name in ("refine", "network", "pipeline", "shim", "shard", "batch", "band", "post",
                "image", "train", "band_train"):
        return importlib.import_module("." + name, __name__)
    raise AttributeError(name)
