"""CPU restatement of the stroke-to-seed ray march (float32 numpy).  TEST
INFRASTRUCTURE ONLY: the checker of jfc_stroke_to_seeds.

Follows graphcut_compute_visibility (src/QVisualizer/cl/GraphCut/
graphcut_render_ray_casting.cl:275-346) with its helpers intersectRay and
backProject (:27-60) and saveMask (:259-273): rays from the inverse
view-projection, slab intersection with [-box, box], non-uniform steps,
trilinear volume samples and a linear transfer-function lookup as OpenCL's
CLK_FILTER_LINEAR | CLK_ADDRESS_CLAMP_TO_EDGE samplers define them (texel
centres at i + 0.5), front-to-back opacity with early termination, and the 8
voxels around every sample more opaque than alpha."""
import numpy as np

f32 = np.float32


def _tex3(vol, x, y, z):
    d, h, w = vol.shape
    x, y, z = f32(x - f32(0.5)), f32(y - f32(0.5)), f32(z - f32(0.5))
    fx, fy, fz = np.floor(x), np.floor(y), np.floor(z)
    ax, ay, az = f32(x - fx), f32(y - fy), f32(z - fz)
    cl = lambda v, n: int(min(max(int(v), 0), n - 1))
    x0, x1 = cl(fx, w), cl(fx + 1, w)
    y0, y1 = cl(fy, h), cl(fy + 1, h)
    z0, z1 = cl(fz, d), cl(fz + 1, d)
    one = f32(1)
    c00 = vol[z0, y0, x0] * (one - ax) + vol[z0, y0, x1] * ax
    c10 = vol[z0, y1, x0] * (one - ax) + vol[z0, y1, x1] * ax
    c01 = vol[z1, y0, x0] * (one - ax) + vol[z1, y0, x1] * ax
    c11 = vol[z1, y1, x0] * (one - ax) + vol[z1, y1, x1] * ax
    c0 = c00 * (one - ay) + c10 * ay
    c1 = c01 * (one - ay) + c11 * ay
    return f32(c0 * (one - az) + c1 * az)


def _tex1(tf, u):
    n = tf.shape[0]
    x = f32(u * f32(n) - f32(0.5))
    fx = np.floor(x)
    a = f32(x - fx)
    i0, i1 = min(max(int(fx), 0), n - 1), min(max(int(fx) + 1, 0), n - 1)
    return tf[i0] * (f32(1) - a) + tf[i1] * a


def stroke_to_seeds(vol, tf, mask, m, box, samples, ratio, step_scale, window_width, window_level, alpha, label,
                    seeds):
    """vol (d,h,w) float32, tf (n,4) float32, mask (ih,iw) uint8, m 16 floats
    (column-major inverse view-projection); marks `seeds` (d,h,w) in place."""
    d, h, w = vol.shape
    ih, iw = mask.shape
    m = np.asarray(m, f32)
    box = np.asarray(box, f32)
    wmin, wmax = f32(window_level - window_width / 2), f32(window_level + window_width / 2)
    mx, my, mz = f32(w - 1), f32(h - 1), f32(d - 1)
    for py in range(ih):
        for px in range(iw):
            if not mask[py, px]:
                continue
            u = f32((px + f32(0.5)) / f32(iw) * f32(2) - f32(1))
            v = f32((py + f32(0.5)) / f32(ih) * f32(2) - f32(1))
            bp = lambda z: np.array([u * m[r] + v * m[4 + r] + f32(z) * m[8 + r] + m[12 + r] for r in range(4)], f32)
            a, b = bp(-1.0), bp(0.0)
            o = a[:3] / a[3]
            dr = b[:3] / b[3] - o
            dr = (dr * (f32(1) / np.sqrt(np.sum(dr * dr, dtype=f32)))).astype(f32)
            with np.errstate(divide="ignore", invalid="ignore"):
                inv = (f32(1) / dr).astype(f32)
                t0 = inv * (-box - o)
                t1 = inv * (box - o)
            tn = f32(np.max(np.minimum(t0, t1)))
            tf_ = f32(np.min(np.maximum(t0, t1)))
            if not tn < tf_:
                continue
            tn = max(tn, f32(0))
            s = np.array([mx / 2 / box[0], my / 2 / box[1], mz / 2 / box[2]], f32)
            q = ((o + dr * tn) * s + np.array([mx / 2, my / 2, mz / 2], f32)).astype(f32)
            dd = (dr * s).astype(f32)
            step = f32((tf_ - tn) / f32(samples - 1) * f32(ratio))
            delta = f32(((tf_ - tn) / f32(samples - 1) - step) / f32(samples - 2))
            acc = f32(0)
            for _ in range(samples):
                val = _tex3(vol, q[0], q[1], q[2])
                c = _tex1(tf, min(max(val, wmin), wmax))
                acc = f32(acc + c[3] * f32(step_scale) * step * np.exp(-acc, dtype=f32))
                if acc >= 1:
                    break
                if c[3] > alpha:
                    xs = [int(min(max(np.floor(q[0]) + k, 0), mx)) for k in (0, 1)]
                    ys = [int(min(max(np.floor(q[1]) + k, 0), my)) for k in (0, 1)]
                    zs = [int(min(max(np.floor(q[2]) + k, 0), mz)) for k in (0, 1)]
                    for zz in zs:
                        for yy in ys:
                            for xx in xs:
                                seeds[zz, yy, xx] = label
                q = (q + dd * step).astype(f32)
                step = f32(step + delta)
    return seeds
