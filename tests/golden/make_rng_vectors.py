"""Generates tests/golden/rng_vectors.json: splitmix64 start states and draws of the PatchStereo RNG.

The rule is restated here independently of the oracle, in plain Python integers, from the reference:
  rng_state  crates/dense/src/kernel.rs:247-252 (= patchmatch.cu:122-125):
             mix64(seed ^ mix64(key ^ mix64(level<<48 ^ run<<32 ^ t<<16 ^ half)) ^ pixel)
  rng_next   crates/dense/src/kernel.rs:254-259: state += 0x9e3779b97f4a7c15; ((mix64(state) >> 40) + 1) * 2^-24
  mix64      crates/dense/src/math.rs:41-47 (splitmix64 finaliser)
  hash_bytes crates/dense/src/math.rs:31-39 (FNV-1a 64)
Run: python tests/golden/make_rng_vectors.py
"""
import json
import os

M = (1 << 64) - 1


def mix64(z):
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
    return z ^ (z >> 31)


def rng_state(seed, key, level, run, t, half, pixel):
    tag = ((level << 48) ^ (run << 32) ^ (t << 16) ^ half) & M
    return mix64((seed ^ mix64((key ^ mix64(tag)) & M) ^ pixel) & M)


def rng_next(s):
    s = (s + 0x9E3779B97F4A7C15) & M
    z = mix64(s)
    return s, ((z >> 40) + 1) / 16777216.0  # exact in binary32: 24-bit integer times 2^-24


def fnv1a(b):
    h = 0xCBF29CE484222325
    for x in b:
        h ^= x
        h = (h * 0x100000001B3) & M
    return h


def main():
    cases = []
    seed = 0x005E_ED0F_DE75  # DensifyOptions::base seed (crates/dense/src/params.rs:427)
    for name in ["synth_0_0.png", "synth_1_2.png", "IMG_0001.JPG", ""]:
        key = fnv1a(name.encode())
        for (level, run, t, half, pixel) in [(0, 1, 0xFFFF, 0, 0), (2, 3, 4, 1, 123456), (1, 7, 0, 0, 2073599)]:
            s = rng_state(seed, key, level, run, t, half, pixel)
            draws = []
            st = s
            for _ in range(5):
                st, u = rng_next(st)
                draws.append(u)
            cases.append({"name": name, "key": key, "seed": seed, "level": level, "run": run, "t": t, "half": half,
                          "pixel": pixel, "state": s, "draws": draws, "final": st})
    mixes = [[z, mix64(z)] for z in [0, 1, 0x9E3779B97F4A7C15, M, 0x0123456789ABCDEF]]
    out = {"cases": cases, "mix64": mixes}
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "rng_vectors.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
