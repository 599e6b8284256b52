"""Host parts of the headless volume view: the orbit camera, the PPM writer and
the oracle's restatement of the shader (src/render/Vis3D.cpp:30-78)."""
import numpy as np

from myfluidsimulation_b200.render import orbit_camera, write_ppm


def glm_like(yaw, pitch, radius, target, w, h):
    """perspective(45 deg, w/h, 0.01, 10) and lookAt(eye, target, +y) as glm builds them."""
    t = np.asarray(target, np.float64)
    eye = t + radius * np.array([np.cos(pitch) * np.cos(yaw), np.sin(pitch), np.cos(pitch) * np.sin(yaw)])
    f = (t - eye) / np.linalg.norm(t - eye)
    s = np.cross(f, [0, 1, 0])
    s /= np.linalg.norm(s)
    u = np.cross(s, f)
    V = np.eye(4)
    V[0, :3], V[1, :3], V[2, :3] = s, u, -f
    V[:3, 3] = [-s @ eye, -u @ eye, f @ eye]
    th = np.tan(np.radians(45.0) / 2)
    P = np.zeros((4, 4))
    P[0, 0], P[1, 1] = 1 / (w / h * th), 1 / th
    P[2, 2], P[2, 3], P[3, 2] = -(10.01) / 9.99, -2 * 10 * 0.01 / 9.99, -1
    return np.linalg.inv(P @ V), eye


def test_orbit_camera_matches_glm_construction():
    for yaw, pitch, radius, (w, h) in [(0.0, 0.3, 2.5, (1280, 720)), (1.1, -0.4, 3.0, (64, 64)),
                                       (-2.0, 0.9, 1.7, (300, 500))]:
        inv, cam = orbit_camera(yaw, pitch, radius, (0.5, 0.5, 0.5), w, h)
        want, eye = glm_like(yaw, pitch, radius, (0.5, 0.5, 0.5), w, h)
        np.testing.assert_allclose(cam, eye, rtol=1e-6, atol=1e-6)
        np.testing.assert_allclose(inv.reshape(4, 4).T, want, rtol=1e-5, atol=1e-5 * np.abs(want).max())


def test_oracle_frame_basics(oracle):
    inv, cam = orbit_camera(width=48, height=32)
    # below the threshold everywhere: every ray through the box ends black and opaque-less
    f = np.zeros((6, 7, 8), np.float32)
    img, ns = oracle.raymarch(f, inv, cam, 0.01, 150.0, 0.15, 48, 32)
    clear = np.array([0.02, 0.02, 0.03, 1.0], np.float32)
    hit = ~np.all(img == clear, axis=2)
    assert hit.any() and (~hit).any() and ns > 0
    assert np.all(img[hit] == np.array([0, 0, 0, 1], np.float32))
    # a strong uniform field: the first sample is already opaque enough to stop by 0.95
    g = np.full((6, 7, 8), 0.01, np.float32)          # scaled 1.5 -> |s| clamps to 1, alpha 1
    img2, ns2 = oracle.raymarch(g, inv, cam, 0.01, 150.0, 0.15, 48, 32)
    assert ns2 == int(hit.sum())                       # one sample per ray that enters the box
    np.testing.assert_allclose(img2[hit][:, :3], np.tile([1.0, 0.1, 0.0], (int(hit.sum()), 1)), atol=1e-6)


def test_ppm_writer(tmp_path):
    img = np.zeros((2, 3, 4), np.float32)
    img[0, 0, :3] = [1.0, 0.5, -1.0]      # bottom-left in GL order
    img[1, 2, :3] = [2.0, 0.25, 0.0]      # top-right
    p = tmp_path / "a.ppm"
    write_ppm(p, img)
    data = p.read_bytes()
    head = b"P6\n3 2\n255\n"
    assert data.startswith(head)
    px = np.frombuffer(data[len(head):], np.uint8).reshape(2, 3, 3)
    assert px[1, 0].tolist() == [255, 128, 0]          # written bottom row last
    assert px[0, 2].tolist() == [255, 64, 0]
