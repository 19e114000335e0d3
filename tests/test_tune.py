"""The tuner's host side, without a GPU: pinning a choice, and the refusals for choices that no
kernel compiles."""
import pytest

from shaderous_b200 import tune


def test_pins_and_unpins():
    try:
        tune.pin("uniform_sweep", 0, 16)      # the 2D march at 16 rows a CTA (or 16 z planes in 3D)
        tune.pin("uniform_sweep", 0, 0)       # 2D: the tile form
        tune.pin("amr_assemble", 6, 1)        # the split form side by side
        tune.pin("amr_assemble_bins", 3, 4)
        tune.pin("amr_sweep", 0, 2)
    finally:
        for k in ("uniform_sweep", "amr_assemble", "amr_assemble_bins", "amr_sweep"):
            tune.pin(k, None)


@pytest.mark.parametrize("kernel,variant,per_sm", [
    ("uniform_sweep", 1, 16),       # the sweep has one variant
    ("uniform_sweep", 0, 2000),     # a depth beyond 1024
    ("uniform_sweep", 0, -1),
    ("amr_assemble", 7, 4),         # variants 0-6
    ("amr_assemble", 3, 64),        # at most 32 CTAs per SM
    ("amr_assemble_bins", 2, 4),    # the substeps' assemble: 1 or 3
    ("amr_fine_flux", 1, 8),
])
def test_refuses_choices_no_kernel_has(kernel, variant, per_sm):
    with pytest.raises(ValueError):
        tune.pin(kernel, variant, per_sm)
