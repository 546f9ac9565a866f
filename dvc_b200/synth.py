"""Seeded synthetic test sequences for the Wyner-Ziv decoder.

The reference's own test sequences (foreman, soccer, coastguard, hall) are not
available, so these generators stand in for them with the shapes, sizes and
value distributions of the benchmark configurations:

* ``qcif``: 176x144 luma, a texture of 6 random 2-D sinusoids (periods 4-40 px,
  amplitudes summing to 80) around 128, plus N(0, 3) noise, clipped to [0, 255].
  The frame translates by a seeded integer velocity in [-3, 3] px/frame and two
  32x32 textured rectangles move independently at velocities in [-4, 4].
* ``cif``: 352x288, sinusoid periods scaled x2 (8-80 px), four 48x48 objects.
* ``cif_fast``: 352x288, global velocity in [-8, 8], six objects of 16-64 px
  moving at [-10, 10] px/frame.
* ``qcif_still`` / ``cif_still``: as ``qcif`` / ``cif`` with a still background
  (no global motion) and N(0, 1) noise, so that the encoder's skip test (8x8
  block MSE against the past frame below 10) finds skip blocks.

Chroma planes are constant 128 (4:2:0).  Key frames are the original frames plus
N(0, 2) noise, rounded and clipped; the key-frame info file carries a fixed
4000 bits per frame (the per_frame_stat format parsed by the reference at
DvcDec/src/frame.cpp:197-247).
"""
import numpy as np

SHAPES = {"qcif": (176, 144), "cif": (352, 288), "cif_fast": (352, 288), "qcif_still": (176, 144),
          "cif_still": (352, 288)}


def _params(kind):
    if kind == "qcif":
        return dict(per=(4.0, 40.0), vel=3, n_obj=2, obj=(32, 32), ovel=4)
    if kind == "cif":
        return dict(per=(8.0, 80.0), vel=3, n_obj=4, obj=(48, 48), ovel=4)
    if kind == "cif_fast":
        return dict(per=(8.0, 80.0), vel=8, n_obj=6, obj=(16, 64), ovel=10)
    if kind == "qcif_still":
        return dict(per=(4.0, 40.0), vel=0, n_obj=2, obj=(32, 32), ovel=4, noise=1.0)
    if kind == "cif_still":
        return dict(per=(8.0, 80.0), vel=0, n_obj=4, obj=(48, 48), ovel=4, noise=1.0)
    raise ValueError(kind)


def make_sequence(kind, n_frames, seed):
    """Return (original, key) luma sequences, uint8 arrays of shape (T, H, W).

    The background is an analytic texture (128 plus six sinusoids) on an
    unbounded canvas; each frame evaluates it only where it is seen (the
    translated frame window and the objects' patches), so long sequences with
    fast motion need no canvas in memory."""
    w, h = SHAPES[kind]
    p = _params(kind)
    rng = np.random.default_rng(seed)
    margin = (p["vel"] + p["ovel"]) * n_frames + 128
    th, tw = h + 2 * margin, w + 2 * margin
    amps = rng.dirichlet(np.ones(6)) * 80.0
    waves = []
    for a in amps:
        per = rng.uniform(*p["per"])
        ang = rng.uniform(0, np.pi)
        ph = rng.uniform(0, 2 * np.pi)
        waves.append((a, per, ang, ph))

    def tex(y0, x0, hh, ww):
        """Texture over rows y0..y0+hh-1 and columns x0..x0+ww-1 of the canvas."""
        yy, xx = np.mgrid[y0:y0 + hh, x0:x0 + ww].astype(np.float64)
        t = np.full((hh, ww), 128.0)
        for a, per, ang, ph in waves:
            t += a * np.sin(2 * np.pi * (xx * np.cos(ang) + yy * np.sin(ang)) / per + ph)
        return t

    vx, vy = rng.integers(-p["vel"], p["vel"] + 1, 2)
    objs = []
    for _ in range(p["n_obj"]):
        size = int(rng.integers(p["obj"][0], p["obj"][1] + 1))
        objs.append(dict(
            size=size,
            x=int(rng.integers(0, w - size)), y=int(rng.integers(0, h - size)),
            vx=int(rng.integers(-p["ovel"], p["ovel"] + 1)),
            vy=int(rng.integers(-p["ovel"], p["ovel"] + 1)),
            # texture patch the object carries, taken away from the background window
            sx=int(rng.integers(0, tw - size)), sy=int(rng.integers(0, th - size)),
        ))
    for o in objs:
        o["patch"] = tex(o["sy"], o["sx"], o["size"], o["size"])
    orig = np.empty((n_frames, h, w), np.uint8)
    key = np.empty((n_frames, h, w), np.uint8)
    for t in range(n_frames):
        ox, oy = margin + vx * t, margin + vy * t
        f = tex(oy, ox, h, w)
        for o in objs:
            s = o["size"]
            # objects wrap around inside the frame so they never leave it
            x = (o["x"] + o["vx"] * t) % (w - s)
            y = (o["y"] + o["vy"] * t) % (h - s)
            f[y:y + s, x:x + s] = o["patch"]
        f = np.clip(np.rint(f + rng.normal(0.0, p.get("noise", 3.0), f.shape)), 0, 255)
        k = np.clip(np.rint(f + rng.normal(0.0, 2.0, f.shape)), 0, 255)
        orig[t] = f.astype(np.uint8)
        key[t] = k.astype(np.uint8)
    return orig, key


def write_yuv420(path, frames):
    """Write luma frames as planar YUV 4:2:0 with constant-128 chroma."""
    t, h, w = frames.shape
    chroma = np.full(h * w // 2, 128, np.uint8).tobytes()
    with open(path, "wb") as f:
        for i in range(t):
            f.write(frames[i].tobytes())
            f.write(chroma)


def read_y(path, w, h, n_frames=None, y_only=False):
    """Read the luma planes of a YUV 4:2:0 file (or a Y-only file)."""
    data = np.fromfile(path, np.uint8)
    per = w * h if y_only else w * h * 3 // 2
    n = len(data) // per if n_frames is None else n_frames
    return np.stack([data[i * per:i * per + w * h].reshape(h, w) for i in range(n)])


def write_frame_stat(path, n_frames, bits=4000, qp=30, psnr=40.0):
    with open(path, "w") as f:
        for t in range(n_frames):
            f.write(f"FrameNo: {t} Y_bits: {bits} UV_bits: 0 QP: {qp} Y_psnr: {psnr:.2f}\n")
