"""Learned warm start for GraphFlood: a 4-level U-Net on hand-written BF16
tensor-core convolutions predicts the initial water depth, and the plain
GraphFlood iteration continues from it.  No reference counterpart."""
from .unet import UNet, LAYERS
from .warm import features, make_dataset, train, predict_h0

__all__ = ["UNet", "LAYERS", "features", "make_dataset", "train", "predict_h0"]
