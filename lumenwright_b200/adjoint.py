"""The differentiable form: parameters theta of an hq frame, an L2 image loss, its gradient by the
library's path-replay adjoint, and paired central finite differences to check it.

theta, as one flat FP64 vector:
  - ``albedo``: 64 block-texture slots x 16x16 texels x RGB linear albedos (49,152 values). Slot i
    is the i-th texture of the atlas (``synth.TEXTURES``); its 16x16 texels, and the one-texel
    border the atlas packer copies from their edge, map to the slot's parameters. At the nominal
    theta each value is the texel's decoded colour (gamma_to_linear of its bytes), so the forward
    image is the plain renderer's. Slots past the atlas's textures are parameters no texel reads.
  - ``emitter``: 32 emitter-group intensities (nominal 1), multiplying the frame's emitter
    intensity for the emitters whose voxel hashes to the group.
  - ``sky``: sun azimuth and altitude (radians) and Preetham turbidity. They set the frame's sun
    direction and Chunky's sky (`hq_params`, crates/lumenwright/src/request.rs:1153-1225, and
    `Preetham::new`, crates/lumenwright/src/render/sky.rs:666-742); the device builds the sky cache.

The kernel returns the gradient with respect to the sun direction vector and to every sky-cache
entry; the host chains them to (azimuth, altitude, turbidity) with the analytic derivative of the
direction and the Jacobian of the cache, taken by FP64 central differences of an FP64 statement of
the cache builder (`build_sky_cache`, crates/lumenwright-kernel/src/integrator.rs:133-148, with
`preetham_radiance` :44-74 and `rgb_to_hsl` :79-104).

The differentiation workload: the 8x8-chunk world with emitters, 512x288, 64 spp, 4 bounces,
Chunky's sky at tick 4000 (altitude from the celestial angle) with the sun turned to azimuth 0.3
rad. The reference's suns move in the x-y plane, where `sample_sun`'s cone frame (the `onb` of
math.rs:348-356) switches sign at sun.z = 0; a finite difference in azimuth across that switch
compares different cone samples, so the nominal sun sits off it.
"""

import math
from dataclasses import dataclass

import numpy as np

from . import request as R
from . import sky as SK
from . import synth as S
from .hqbuild import build_hq

F32 = np.float32
SLOTS = 64
TEXELS = 256
N_ALBEDO = SLOTS * TEXELS * 3
GROUPS = 32
N_THETA = N_ALBEDO + GROUPS + 3
SKY_NAMES = ("azimuth", "altitude", "turbidity")


def texel_parameters(atlas: S.Atlas, gamma: np.ndarray):
    """(texel_param per atlas texel, nominal albedo (SLOTS * 256, 3)) for the atlas's textures."""
    h, w = atlas.pixels.shape
    tp = np.full((h, w), -1, np.int32)
    albedo = np.zeros((SLOTS * TEXELS, 3), np.float32)
    for i, name in enumerate(S.TEXTURES[:SLOTS]):
        sp = atlas.sprites[name]
        if (sp.w, sp.h) != (16, 16):
            continue
        ys, xs = np.mgrid[-1:17, -1:17]
        u, v = np.clip(xs, 0, 15), np.clip(ys, 0, 15)
        ay, ax = sp.y + ys, sp.x + xs
        ok = (ay >= 0) & (ay < h) & (ax >= 0) & (ax < w)
        tp[ay[ok], ax[ok]] = (i * TEXELS + v * 16 + u)[ok]
        px = atlas.pixels[sp.y:sp.y + 16, sp.x:sp.x + 16].astype(np.uint32).ravel()
        albedo[i * TEXELS:(i + 1) * TEXELS] = np.stack(
            [gamma[px & 0xFF], gamma[(px >> 8) & 0xFF], gamma[(px >> 16) & 0xFF]], -1)
    return tp.ravel(), albedo


def sun_vector(az: float, alt: float) -> np.ndarray:
    return np.array([math.cos(alt) * math.cos(az), math.sin(alt), math.cos(alt) * math.sin(az)])


def sun_vector_jacobian(az: float, alt: float) -> np.ndarray:
    """d sun_vector / d (azimuth, altitude), shape (3, 2)."""
    return np.array([[-math.cos(alt) * math.sin(az), -math.sin(alt) * math.cos(az)],
                     [0.0, math.cos(alt)],
                     [math.cos(alt) * math.cos(az), -math.sin(alt) * math.sin(az)]])


def sky_cache_f64(az: float, alt: float, turbidity: float, n: int = SK.SKY_CACHE_RESOLUTION) -> np.ndarray:
    """Chunky's sky cache of a sun at (az, alt) and a turbidity, in FP64: (n+1)^2 x (h, s, l)."""
    pre = SK.Preetham(sun_vector(az, alt), turbidity)
    sun, zen, perez = pre.sun64, pre.zenith64, pre.perez64
    m = n + 1
    i, j = np.divmod(np.arange(m * m), m)
    th = 2.0 * math.pi * i / n
    ph = 2.0 * math.pi * (j / (2.0 * n) - 0.25)
    r = np.abs(np.cos(ph))
    d = np.stack([np.cos(th) * r, np.sin(ph), np.sin(th) * r], -1)
    cos_theta = np.maximum(d[:, 1], 0.0)
    cos_gamma = np.clip(d @ sun, -1.0, 1.0)
    gamma = np.arccos(cos_gamma)
    with np.errstate(divide="ignore", over="ignore", invalid="ignore"):
        pz = []
        for k in range(3):
            a = np.where(cos_theta > 0.0, perez[0, k] * np.exp(perez[1, k] / np.where(cos_theta > 0, cos_theta, 1.0)), 0.0)
            pz.append((1.0 + a) * (1.0 + perez[2, k] * np.exp(perez[3, k] * gamma) + perez[4, k] * cos_gamma ** 2))
        x, y, lum = zen[0] * pz[0], zen[1] * pz[1], zen[2] * pz[2]
        f = np.where(y > 5e-8, lum / np.where(y > 5e-8, y, 1.0), 0.0)
    cx, cy, cz = x * f, lum, (1.0 - x - y) * f
    rgb = np.stack([2.3706743 * cx - 0.9000405 * cy - 0.4706338 * cz, -0.513885 * cx + 1.4253036 * cy + 0.0885814 * cz,
                    0.0052982 * cx - 0.0146949 * cy + 1.0093968 * cz], -1) * 0.045
    rgb = np.where((y > 5e-8)[:, None], rgb, 0.0)
    c = np.clip(rgb, 0.0, 1.0)
    cmax, cmin = c.max(1), c.min(1)
    delta = cmax - cmin
    light = (cmax + cmin) / 2.0
    sd = np.where(delta == 0.0, 1.0, delta)
    hue = np.where(cmax == c[:, 0], np.fmod((c[:, 1] - c[:, 2]) / sd, 6.0) / 6.0,
                   np.where(cmax == c[:, 1], ((c[:, 2] - c[:, 0]) / sd + 2.0) / 6.0, ((c[:, 0] - c[:, 1]) / sd + 4.0) / 6.0))
    hue = np.where(delta == 0.0, 0.0, hue)
    den = 1.0 - np.abs(2.0 * light - 1.0)
    sat = np.where(delta < 5e-8, 0.0, delta / np.where(den == 0.0, 1.0, den))
    return np.stack([hue, sat, light], -1).ravel()


def sky_cache_jacobian(az: float, alt: float, turbidity: float, h: float = 1e-6) -> np.ndarray:
    """d sky_cache_f64 / d (azimuth, altitude, turbidity), shape (entries, 3), FP64 central
    differences."""
    x0 = np.array([az, alt, turbidity])
    cols = []
    for k in range(3):
        e = np.zeros(3)
        e[k] = h
        cols.append((sky_cache_f64(*(x0 + e)) - sky_cache_f64(*(x0 - e))) / (2.0 * h))
    return np.stack(cols, -1)


@dataclass
class Split:
    albedo: np.ndarray  # (SLOTS * 256, 3) float32
    emitter: np.ndarray  # (32,) float32
    sky: np.ndarray  # (3,) float64


def split(theta: np.ndarray) -> Split:
    return Split(theta[:N_ALBEDO].reshape(-1, 3).astype(F32), theta[N_ALBEDO:N_ALBEDO + GROUPS].astype(F32),
                 theta[N_ALBEDO + GROUPS:].astype(np.float64))


class DiffProblem:
    """An L2 loss between the forward image at theta and a target image, on one context.

    ``theta0`` is the nominal parameter vector; ``target`` is rendered at ``theta0`` plus seeded
    N(0, sigma) noise on every parameter (albedos kept >= 0), with another sample seed."""

    def __init__(self, ctx, width=512, height=288, spp=64, chunks=8, bounces=4, time=4000, azimuth=0.3,
                 world_seed=1, target_seed=5, sigma=0.05, eye=(32.0, 100.0, 32.0), look=(0.0, 64.0, 0.0)):
        from .native import gamma_table
        self.ctx = ctx
        self._pool = None  # the host thread gradient() computes the sky Jacobian on
        self.width, self.height, self.spp, self.bounces = width, height, spp, bounces
        world = S.generate_world(chunks, world_seed, emitters=True)
        atlas = S.build_atlas(world_seed)
        self.hq = build_hq(world, atlas)
        ctx.upload_hq_scene(self.hq)
        self.texel_param, albedo0 = texel_parameters(atlas, gamma_table())
        yaw, pitch = R.Camera.look_at(eye, look)
        self.cam = R.Camera(eye, float(yaw), float(pitch), 70.0)
        self.eye = [F32(eye[i] - world.origin[i]) for i in range(3)]
        sun = SK.sun_direction_from_angle(SK.celestial_angle(time)).astype(np.float64)
        alt = math.asin(max(-1.0, min(1.0, float(sun[1]))))
        self.intensity = SK.default_emitter_intensity(False, F32(1.0))
        self.theta0 = np.concatenate([albedo0.astype(np.float64).ravel(), np.ones(GROUPS), [azimuth, alt, 2.5]])
        rng = np.random.default_rng(target_seed)
        t = self.theta0 + rng.normal(0.0, sigma, N_THETA)
        t[:N_ALBEDO] = np.maximum(t[:N_ALBEDO], 0.0)
        self.theta_target = t
        self.target = self.forward(t, seed=1)

    def frame(self, sky3, seed=0):
        """(params, sky cache) of the sky parameters (azimuth, altitude, turbidity)."""
        az, alt, tb = (float(x) for x in sky3)
        sun = SK.normalize32(sun_vector(az, alt))
        p = R.hq_params(self.width, self.height, self.hq, self.eye, self.cam, SK.hq_sky(sun), spp_seed=seed,
                        max_bounces=self.bounces, emitter_intensity=self.intensity, turbidity=tb)
        cache = self.ctx.build_sky_cache(p, int(p["misc_f"][2]))
        return p, cache

    def _args(self, theta, seed=0, frame=None):
        sp = split(theta)
        p, cache = frame or self.frame(sp.sky, seed)
        return (p, cache, sp.albedo, self.texel_param, sp.emitter)

    def forward(self, theta, seed=0):
        """The FP64 mean image at theta, (h, w, 3)."""
        return self.ctx.adjoint_forward(*self._args(theta, seed), self.spp)

    def loss(self, image):
        return float(np.sum((image - self.target) ** 2))

    def gradient(self, theta):
        """(loss, d loss / d theta) at theta by the adjoint. The sky cache's Jacobian is computed on
        a host thread while the device runs the forward and backward passes (the library's calls
        release the interpreter lock)."""
        args = self._args(theta)
        sp = split(theta)
        az, alt, tb = sp.sky
        if self._pool is None:
            from concurrent.futures import ThreadPoolExecutor
            self._pool = ThreadPoolExecutor(max_workers=1)
        job = self._pool.submit(sky_cache_jacobian, az, alt, tb)
        image = self.ctx.adjoint_forward(*args, self.spp)
        g = self.ctx.adjoint_backward(*args, self.spp, 2.0 * (image - self.target))
        j_cache = job.result()
        g_sky = g["sky"][:j_cache.shape[0]] @ j_cache
        g_sky[:2] += g["sun_dir"] @ sun_vector_jacobian(az, alt)
        out = np.concatenate([g["albedo"].ravel(), g["emitter_scale"], g_sky])
        return self.loss(image), out

    def finite_difference(self, theta, k, h=1e-3):
        """Central difference of the loss in parameter k (paired samples, nominal roulette and shadow
        rays): (loss(theta + h e_k) - loss(theta - h e_k)) / (2 h), with the step the FP32 parameter
        actually takes."""
        tp, tm = theta.copy(), theta.copy()
        tp[k] += h
        tm[k] -= h
        if k < N_ALBEDO + GROUPS:
            h_eff = (float(F32(tp[k])) - float(F32(tm[k]))) / 2.0
            shared = self.frame(split(theta).sky)
            fp = fm = shared
        else:
            h_eff = h
            fp, fm = self.frame(split(tp).sky), self.frame(split(tm).sky)
        nominal = self._args(theta)
        diff, mean = self.ctx.adjoint_fd(self._args(tp, frame=fp), self._args(tm, frame=fm), nominal, self.spp)
        return float(np.sum(diff * 2.0 * (mean - self.target))) / (2.0 * h_eff)

    def check_indices(self, n=256, seed=11):
        """The parameters a check draws: the 3 sky parameters, the 32 emitter groups and the rest
        albedo entries drawn without replacement from the atlas's textures (seeded)."""
        rng = np.random.default_rng(seed)
        used = np.unique(self.texel_param[self.texel_param >= 0])
        entries = (used[:, None] * 3 + np.arange(3)[None]).ravel()
        k = max(0, n - 3 - GROUPS)
        alb = np.sort(rng.choice(entries, size=min(k, entries.size), replace=False))
        return np.concatenate([alb, N_ALBEDO + np.arange(GROUPS), N_ALBEDO + GROUPS + np.arange(3)]).astype(np.int64)


def name_of(k: int) -> str:
    if k < N_ALBEDO:
        slot, rem = divmod(k, TEXELS * 3)
        texel, ch = divmod(rem, 3)
        tex = S.TEXTURES[slot] if slot < len(S.TEXTURES) else f"slot{slot}"
        return f"albedo[{tex}:{texel % 16},{texel // 16}:{'rgb'[ch]}]"
    if k < N_ALBEDO + GROUPS:
        return f"emitter[{k - N_ALBEDO}]"
    return SKY_NAMES[k - N_ALBEDO - GROUPS]


def check(problem: DiffProblem, indices, h=1e-3):
    """Adjoint against central differences on `indices`: a list of dicts per parameter."""
    loss, g = problem.gradient(problem.theta0)
    rows = []
    for k in indices:
        fd = problem.finite_difference(problem.theta0, int(k), h)
        ad = float(g[k])
        rows.append({"index": int(k), "name": name_of(int(k)), "adjoint": ad, "fd": fd,
                     "rel": abs(ad - fd) / max(abs(ad), abs(fd), 1e-300)})
    return loss, g, rows


def main(argv=None):
    """Runs the check on the differentiation workload and writes a JSON report."""
    import argparse
    import json
    import time

    from .native import Context
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--width", type=int, default=512)
    ap.add_argument("--height", type=int, default=288)
    ap.add_argument("--spp", type=int, default=64)
    ap.add_argument("--params", type=int, default=256)
    ap.add_argument("--h", type=float, default=1e-3)
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    ctx = Context(0)
    t0 = time.time()
    prob = DiffProblem(ctx, a.width, a.height, a.spp)
    t1 = time.time()
    loss, g, rows = check(prob, prob.check_indices(a.params), a.h)
    t2 = time.time()
    fd = np.array([r["fd"] for r in rows])
    rel = np.array([r["rel"] for r in rows])
    report = {"workload": f"{a.width}x{a.height}, {a.spp} spp, 8x8 chunks with emitters, 4 bounces, Chunky sky",
              "h": a.h, "loss": loss, "params": len(rows), "nonzero": int(np.count_nonzero(fd)),
              "max_rel": float(rel.max()), "median_rel": float(np.median(rel)),
              "within_1e-3": int(np.count_nonzero(rel <= 1e-3)), "setup_s": t1 - t0, "check_s": t2 - t1,
              "rows": rows}
    text = json.dumps(report, indent=1)
    if a.out:
        with open(a.out, "w") as f:
            f.write(text)
    print(json.dumps({k: v for k, v in report.items() if k != "rows"}))
    ctx.close()


if __name__ == "__main__":
    main()
