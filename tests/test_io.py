"""Result files, landmarks and TRE (host side), and the FP64 restatements of the output images."""
import numpy as np
import pytest

from oracle import multiscale as M
from skmimageregistration_b200 import io as IO


@pytest.mark.parametrize("shape,components", [((5, 6, 7), 0), ((6, 7), 0), ((5, 6, 7, 3), 1), ((6, 7, 2), 1),
                                              ((5, 6, 7, 3, 3), 2)])
@pytest.mark.parametrize("binary", [True, False])
def test_vtk_round_trip(tmp_path, shape, components, binary):
    rng = np.random.default_rng(1)
    a = rng.normal(size=shape)
    D = len(shape) - components
    sp, og = (0.5, 1.25, 2.0)[:D], (-3.0, 4.5, 0.25)[:D]
    p = str(tmp_path / "a.vtk")
    IO.write_vtk(p, a, sp, og, components=components, dtype="double", binary=binary)
    b, sp2, og2 = IO.read_vtk(p)
    assert b.reshape(a.shape).shape == a.shape and np.array_equal(b.reshape(a.shape), a)
    assert sp2 == sp and og2 == og


def test_vtk_header_and_big_endian_float(tmp_path):
    p = str(tmp_path / "s.vtk")
    img = np.arange(24, dtype=np.float64).reshape(2, 3, 4)
    IO.write_vtk(p, img, (1.0, 2.0, 3.0))
    raw = open(p, "rb").read()
    head = raw[:raw.index(b"LOOKUP_TABLE default\n") + len(b"LOOKUP_TABLE default\n")].decode()
    assert head.startswith("# vtk DataFile Version 3.0\n")
    assert "BINARY\nDATASET STRUCTURED_POINTS\nDIMENSIONS 4 3 2\n" in head
    assert "POINT_DATA 24\nSCALARS scalars float 1\n" in head
    body = raw[len(head):len(head) + 24 * 4]
    assert np.array_equal(np.frombuffer(body, ">f4"), img.reshape(-1).astype(np.float32))


def test_read_landmarks(tmp_path):
    p = tmp_path / "lm.vtk"
    p.write_text("# vtk DataFile Version 3.0\n# comment\nPOINTS 3 float\n1 2 3 4 5 6\n7 8 9\n")
    pts = IO.read_landmarks(str(p), 3)
    assert np.array_equal(pts, [[1, 2, 3], [4, 5, 6], [7, 8, 9]])
    assert np.array_equal(IO.read_landmarks(str(p), 2), [[1, 2], [4, 5], [7, 8]])
    p.write_text("POINTS 4 float\n1 2 3\n")
    with pytest.warns(UserWarning):
        IO.read_landmarks(str(p), 3)


def test_target_registration_error():
    u = np.zeros((10, 11, 12, 3))
    u[...] = (0.5, -1.0, 2.0)
    moving = np.array([[3.0, 4.0, 5.0], [1.0, 1.0, 1.0]])
    fixed = moving + (0.5, -1.0, 2.0)
    assert IO.target_registration_error(u, None, None, fixed, moving) == pytest.approx(0.0, abs=1e-14)
    # a point outside the field is not moved
    far = np.array([[100.0, 0.0, 0.0]])
    assert IO.target_registration_error(u, None, None, far + 1.0, far) == pytest.approx(np.sqrt(3.0))
    assert IO.target_registration_error(u, None, None, fixed, moving[:1]) == -1.0
    # linear interpolation between texels
    v = np.zeros((1, 1, 4, 3))
    v[0, 0, :, 0] = [0.0, 1.0, 2.0, 3.0]
    assert IO.target_registration_error(v, None, None, [[1.5 + 1.5, 0, 0]], [[1.5, 0, 0]]) == pytest.approx(0.0)


def test_warp_restatement_properties():
    rng = np.random.default_rng(2)
    img = rng.random((9, 10))
    zero = np.zeros((9, 10, 2))
    g = ((1.0, 1.0), (0.0, 0.0))
    assert np.max(np.abs(M.warp_image(img, zero, *g, *g, order=3) - img)) < 1e-13   # interpolating spline
    assert np.array_equal(M.warp_image(img, zero, *g, *g, order=1), img)
    # an integer shift by one texel along x moves the image; the last column leaves the image
    shift = np.zeros((9, 10, 2))
    shift[..., 0] = 1.0
    w = M.warp_image(img, shift, *g, *g, order=1, default_value=-7.0)
    assert np.array_equal(w[:, :-1], img[:, 1:]) and np.all(w[:, -1] == -7.0)
    # cubic B-spline interpolation reproduces a linear ramp away from the mirrored borders (whose
    # influence decays like (2 - sqrt(3))^distance)
    ramp = np.broadcast_to(np.arange(60.0) * 0.5, (6, 60)).copy()
    sub = np.zeros((6, 60, 2))
    sub[..., 0] = 0.37
    w = M.warp_image(ramp, sub, *g, *g, order=3)
    assert np.allclose(w[:, 16:-16], ramp[:, 16:-16] + 0.5 * 0.37, rtol=0, atol=1e-7)


def test_jacobian_restatement_of_an_affine_field():
    A = np.array([[0.1, 0.02, -0.03], [0.0, -0.2, 0.05], [0.04, 0.0, 0.3]])
    z, y, x = np.indices((6, 7, 8), dtype=np.float64)
    sp = (0.5, 1.0, 2.0)
    pts = np.stack([x * sp[0], y * sp[1], z * sp[2]], -1)
    u = pts @ A.T
    J = M.jacobian_determinant(u, sp)
    assert np.allclose(J[1:-1, 1:-1, 1:-1], np.linalg.det(np.eye(3) + A), atol=1e-13)
    assert np.allclose(M.jacobian_determinant(np.zeros((4, 5, 2)), (1, 1)), 1.0)


def test_oracle_restart_reproduces_the_full_run():
    from helpers import smooth_volume
    rng = np.random.default_rng(17)
    ref = smooth_volume(rng, (24, 26)) * 900 + 100
    tar = smooth_volume(rng, (24, 26)) * 900 + 100
    cfg = dict(num_scales=2, sigma_C4=[8, 6], sigma_C0=[16, 12], cp_spacing_scaler=2.0, smoothing_variance=[1.0, 0],
               sampling_rate=[1], neighborhood_sampling=[1], num_function_evaluations=[3, 3], metric="mse",
               initial_step_size=[4000.0], tensor_weights=[0])
    full, best = M.register(ref, tar, (1.0, 1.0), None, cfg)
    lvl0, _ = M.register(ref, tar, (1.0, 1.0), None, dict(cfg, num_scales=1))
    again, best2 = M.register(ref, tar, (1.0, 1.0), None, dict(cfg, restart_at=2), initial_displacement=lvl0)
    assert len(best2) == 1 and best2[0] == best[1]
    assert np.array_equal(again, full)
