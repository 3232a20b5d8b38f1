"""Learned warm start for GraphFlood: a 4-level U-Net on hand-written BF16
tensor-core convolutions predicts the initial water depth, and the plain
GraphFlood iteration continues from it.  No reference counterpart."""
from .unet import UNet, LAYERS
from .warm import (features, kinematic_h0, make_dataset, predict_h0, scenario_tiles, train, warm_start_batch,
                   warm_start_flooder)

__all__ = ["UNet", "LAYERS", "features", "kinematic_h0", "make_dataset", "predict_h0", "scenario_tiles", "train",
           "warm_start_batch", "warm_start_flooder"]
