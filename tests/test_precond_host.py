"""Host logic of the learned preconditioner (no GPU): the image size the
U-Net runs an FWI image at."""
from elastic_isotropic_operators_b200 import precond


def _levels_tma_ok(h, w):
    return all(precond._tma_level_ok(h >> l, w >> l) for l in range(4))


def test_unet_pad_shape_reaches_the_tma_kernels_cheaply_or_keeps_multiples_of_8():
    # the cfg-3 FWI image ([nx][nz] = 3400 x 1000): 24 more columns put every level on the TMA kernels
    assert precond.unet_pad_shape(3400, 1000) == (3400, 1024)
    assert _levels_tma_ok(3400, 1024) and not _levels_tma_ok(3400, 1000)
    # already tileable sizes stay as they are
    for hw in ((256, 256), (136, 520), (1000, 3400), (64, 64)):
        assert precond.unet_pad_shape(*hw) == hw
    # no tileable size within 15 % more pixels: multiples of 8 (the copy-loop kernel takes those)
    assert precond.unet_pad_shape(104, 72) == (104, 72)
    assert precond.unet_pad_shape(101, 70) == (104, 72)
    # the chosen size is never smaller, always a multiple of 8, and tileable whenever it grew past the multiple
    for h in range(8, 300, 13):
        for w in range(8, 300, 17):
            hh, ww = precond.unet_pad_shape(h, w)
            assert hh >= h and ww >= w and hh % 8 == 0 and ww % 8 == 0
            assert hh * ww <= 1.15 * h * w or (hh, ww) == (-(-h // 8) * 8, -(-w // 8) * 8)
            if (hh, ww) != (-(-h // 8) * 8, -(-w // 8) * 8):
                assert _levels_tma_ok(hh, ww)
