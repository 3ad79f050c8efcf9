"""Learned warm start: a BF16 U-Net that maps a dirty image to a starting
image for the plain L-BFGS-B solve (no reference counterpart)."""
