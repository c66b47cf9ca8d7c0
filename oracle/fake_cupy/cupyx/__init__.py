"""cupyx stand-in: scatter_add -> numpy.add.at (sequential index order, f32)."""
import numpy as np


def scatter_add(a, slices, value):
    np.add.at(a, slices, value)
