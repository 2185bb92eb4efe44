"""Generate the golden fixtures from the reference's own compiled code.

Every fixture here is produced by oracle/_ref/libbh_ref.so, i.e. by the
reference's unmodified src/physics/kerr.cpp (physics::kerrPotentials,
physics::kerrStepMino) and the headers it compiles with (kerr.h,
novikov_thorne.h), driven through oracle/ref_shim.cpp. The CPU tests check
the oracle restatement against these files; the GPU tests check the CUDA
library against them. Run in a container that has the reference sources:

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from blackhole_b200._abi import default_scene  # noqa: E402
from oracle.pyoracle import RefLib, build  # noqa: E402

OUT = Path(__file__).resolve().parent
SEED = 20261203

C_CGS = 2.99792458e10
G_CGS = 6.67430e-8
M_SUN = 1.98841e33
UNIT_MASS = C_CGS * C_CGS / G_CGS  # G * mass / c^2 == 1 exactly


def scene_dict(s) -> dict:
    return s.as_dict()


def save(name: str, scene=None, **arrays):
    if scene is not None:
        arrays["scene_json"] = np.array(json.dumps(scene_dict(scene)))
    np.savez_compressed(OUT / name, **arrays)
    print(f"wrote {name} ({(OUT / name).stat().st_size / 1024:.1f} KiB)")


def random_states(rng, n, m_geom_scale=1.0):
    """Seeded states in the region the reference stepper is exercised in."""
    r = rng.uniform(3.0, 60.0, n) * m_geom_scale
    theta = rng.uniform(0.2, np.pi - 0.2, n)
    phi = rng.uniform(0.0, 2 * np.pi, n)
    t = np.zeros(n)
    sr = rng.choice([-1.0, 1.0], n)
    sth = rng.choice([-1.0, 1.0], n)
    e = np.ones(n)
    lz = rng.uniform(-6.0, 6.0, n) * m_geom_scale
    q = rng.uniform(0.0, 40.0, n) * m_geom_scale**2
    return dict(r=r, theta=theta, phi=phi, t=t, sign_r=sr, sign_theta=sth), e, lz, q


def main() -> None:
    build()
    ref = RefLib()
    rng = np.random.default_rng(SEED)

    # --- kerrPotentials / kerrStepMino on seeded states (geometric and CGS) ---
    arrays = {}
    for tag, mass, scale, spin in (("geom", UNIT_MASS, 1.0, 0.9), ("cgs", 10.0 * M_SUN, G_CGS * 10.0 * M_SUN / C_CGS**2, 0.3)):
        st, e, lz, q = random_states(rng, 512, scale)
        a = spin * scale
        pot = ref.potentials(st["r"], st["theta"], mass, a, e, lz, q)
        dlam = rng.uniform(1e-4, 5e-3, 512) / scale  # Mino step scales as 1/length
        one = ref.step_mino(st, mass, a, e, lz, q, dlam, 1)
        hundred = ref.step_mino(st, mass, a, e, lz, q, dlam, 100)
        arrays.update({f"{tag}_mass": np.float64(mass), f"{tag}_a": np.float64(a), f"{tag}_dlam": dlam,
                       f"{tag}_e": e, f"{tag}_lz": lz, f"{tag}_q": q})
        for k, v in st.items():
            arrays[f"{tag}_in_{k}"] = v
        for k, v in pot.items():
            arrays[f"{tag}_pot_{k}"] = v
        for k, v in one.items():
            arrays[f"{tag}_step1_{k}"] = v
        for k, v in hundred.items():
            arrays[f"{tag}_step100_{k}"] = v
    save("kerr_step_ref.npz", **arrays)

    # --- KerrRaytracer::trace: the reference's own equatorial use and general rays ---
    # "cgs": physics::KerrRaytracer(M_sun, a) with its constructor defaults
    # (step 0.02 r_s of Mino time: every ray leaves in one step).
    # "geom": M = 1 units, Mino step 2e-4 from r = 30, escape at 100: long
    # rays with captures, escapes and the reference's turning-point stalls.
    arrays = {}
    for unit in ("cgs", "geom"):
        mass = M_SUN if unit == "cgs" else UNIT_MASS
        m_geom = G_CGS * mass / C_CGS**2
        r_s = 2.0 * m_geom
        for spin_tag, spin in (("a0", 0.0), ("a09", 0.9)):
            tag = f"{unit}_{spin_tag}"
            d = ref.raytracer_defaults(mass, spin * m_geom)
            if unit == "geom":
                d.update(r_escape=100.0, step_size=2e-4)
                r0, max_steps = 30.0, 5000
            else:
                r0, max_steps = 12.0 * r_s, 3000
            n = 96
            b = np.linspace(2.0, 12.0, n) * m_geom
            st = dict(r=np.full(n, r0), theta=np.full(n, 0.5 * np.pi), phi=np.linspace(0, 2 * np.pi, n),
                      t=np.zeros(n), sign_r=-np.ones(n), sign_theta=np.ones(n))
            res = ref.trace_rays(st, np.ones(n), b, np.zeros(n), mass, d["a"], d["r_horizon"], d["r_escape"],
                                 d["step_size"], max_steps)
            arrays[f"{tag}_eq_b"] = b
            for k, v in st.items():
                arrays[f"{tag}_eq_in_{k}"] = v
            for k, v in res.items():
                arrays[f"{tag}_eq_{k}"] = v
            st2, e2, lz2, q2 = random_states(rng, n, m_geom)
            st2["r"] = np.full(n, r0) * rng.uniform(0.5, 1.0, n)
            res2 = ref.trace_rays(st2, e2, lz2, q2, mass, d["a"], d["r_horizon"], d["r_escape"], d["step_size"],
                                  max_steps)
            for k, v in st2.items():
                arrays[f"{tag}_gen_in_{k}"] = v
            arrays[f"{tag}_gen_e"], arrays[f"{tag}_gen_lz"], arrays[f"{tag}_gen_q"] = e2, lz2, q2
            for k, v in res2.items():
                arrays[f"{tag}_gen_{k}"] = v
            for k, v in d.items():
                arrays[f"{tag}_{k}"] = np.float64(v)
            arrays[f"{tag}_mass"] = np.float64(mass)
            arrays[f"{tag}_max_steps"] = np.int32(max_steps)
    save("kerr_trace_ref.npz", **arrays)
    m_geom = G_CGS * M_SUN / C_CGS**2

    # --- image tracer scenes with the reference's compiled potentials ---
    s = default_scene(width=64, height=64)
    save("image_c0_64.npz", s, **ref.trace_pixels(s))

    s = default_scene(width=256, height=256)
    full = ref.trace_pixels(s)
    sub = np.arange(0, 256 * 256, 13, dtype=np.int64)
    save("image_c0_256.npz", s, cls=full["cls"].astype(np.uint8), steps=full["steps"], sub_index=sub,
         sub_r_hit=full["r_hit"][0][sub], sub_phi_hit=full["phi_hit"][0][sub], sub_g=full["g"][0][sub],
         sub_flux=full["flux"][sub], sub_theta_inf=full["theta_inf"][sub], sub_phi_inf=full["phi_inf"][sub])

    s = default_scene(width=64, height=64, potential_form=1)
    save("image_carter_64.npz", s, **ref.trace_pixels(s))

    for tag, spin, inc in (("a0998_i85", 0.998, 85.0), ("a05_i17", 0.5, 17.0)):
        s = default_scene(width=32, height=32, spin=spin, theta_obs=np.deg2rad(inc), integrator=1,
                          max_crossings=3, rtol=1e-8, atol=1e-10)
        save(f"image_dp45_{tag}_32.npz", s, **ref.trace_pixels(s))

    # --- known answers from the reference headers ---
    ka = {}
    for spin in (0.0, 0.3, 0.5, 0.9, 0.998):
        ka[str(spin)] = ref.radii(M_SUN, spin * m_geom)
    ka["m_geom"] = m_geom
    (OUT / "known_answers_ref.json").write_text(json.dumps(ka, indent=1, sort_keys=True) + "\n")
    print("wrote known_answers_ref.json")


if __name__ == "__main__":
    main()
