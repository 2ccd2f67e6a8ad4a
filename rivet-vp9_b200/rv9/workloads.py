"""The benchmark configurations' streams: their definitions and an on-disk
cache.

Every stream comes from the repository's seeded generator and encoder
(rv9.streams, librv9enc.so) the first time it is asked for and is kept as an
IVF file under rivet-vp9_b200/_build/streams/, named by the stream's name and
a digest of its parameters (a changed definition never reads a stale file).
Later reads only parse the IVF, so a caller that finds the cache filled never
loads the generator.

The definitions follow the five benchmark configurations:
  CONFIG1  30 frames 352x288 8-bit 4:2:0, one tile column, q60, golden every 8
  CONFIG2  60 frames 1920x1080 8-bit 4:2:0, 4 tile columns, q40 and q80
  CONFIG3  60 frames 3840x2160 10-bit 4:2:0 and 30 frames 1280x720 12-bit
           4:4:4, q30, 4 tile columns, LAST and GOLDEN references
  CONFIG4  64 independent streams, seeds 0..63, sizes 320x240 .. 1080p, 8/10-bit,
           60 frames, q in [30, 90]
  BATCH_CLASSES  eight size / depth classes (the batched tests' contents)
  SERVE_CLASSES  the contents of the 32-stream serving mix (720p / 1080p /
           2160p at 8 and 10 bits)
"""
import hashlib
import json
import os

from . import containers

_HERE = os.path.dirname(os.path.abspath(__file__))
STREAM_DIR = os.path.join(os.path.dirname(_HERE), "_build", "streams")


def _spec(name, width, height, frames, q, seed, bit_depth=8, chroma=(1, 1), tile_cols_log2=None, golden_interval=8,
          pan=(3, 2), rectangles=12, noise=None, color_space=0):
    if tile_cols_log2 is None:
        tile_cols_log2 = 2 if width >= 1024 else 0
    if noise is None:
        noise = 24 if bit_depth > 8 else 6
    return dict(name=name, width=width, height=height, frames=frames, q=q, seed=seed, bit_depth=bit_depth,
                chroma=tuple(chroma), tile_cols_log2=tile_cols_log2, golden_interval=golden_interval, pan=tuple(pan),
                rectangles=rectangles, noise=noise, color_space=color_space)


CONFIG1 = [_spec("cif_q60", 352, 288, 30, 60, seed=0, tile_cols_log2=0, pan=(2, 1), rectangles=3, noise=8)]
CONFIG2 = [_spec("1080p_q40", 1920, 1080, 60, 40, seed=0), _spec("1080p_q80", 1920, 1080, 60, 80, seed=1)]
CONFIG3 = [_spec("2160p_10bit_q30", 3840, 2160, 60, 30, seed=2, bit_depth=10, noise=24),
           _spec("720p_12bit_444_q30", 1280, 720, 30, 30, seed=3, bit_depth=12, chroma=(0, 0), noise=24)]


def _config4():
    """Configuration 4: 64 independent streams, seeds 0..63, each of a size
    drawn uniformly from {320x240, 640x360, 1280x720, 1920x1080}, 8-bit or
    10-bit with probability 0.5, 4:2:0, 60 frames, base q uniform in
    [30, 90] (the draws from a generator seeded by the stream's seed)."""
    import random
    sizes = [(320, 240), (640, 360), (1280, 720), (1920, 1080)]
    out = []
    for seed in range(64):
        rng = random.Random(7919 * seed + 4)
        w, h = sizes[rng.randrange(4)]
        bd = 10 if rng.random() < 0.5 else 8
        q = rng.randint(30, 90)
        out.append(_spec(f"c4_{seed:02d}_{w}x{h}_{bd}_q{q}", w, h, 60, q, seed=seed, bit_depth=bd))
    return out


CONFIG4 = _config4()
CLASS_FRAMES = 30
BATCH_CLASSES = [
    _spec("b240_8", 320, 240, CLASS_FRAMES, 35, seed=11),
    _spec("b240_10", 320, 240, CLASS_FRAMES, 80, seed=12, bit_depth=10),
    _spec("b360_8", 640, 360, CLASS_FRAMES, 60, seed=13),
    _spec("b360_10", 640, 360, CLASS_FRAMES, 45, seed=14, bit_depth=10),
    _spec("b720_8", 1280, 720, CLASS_FRAMES, 70, seed=15),
    _spec("b720_10", 1280, 720, CLASS_FRAMES, 40, seed=16, bit_depth=10),
    _spec("b1080_8", 1920, 1080, CLASS_FRAMES, 55, seed=17),
    _spec("b1080_10", 1920, 1080, CLASS_FRAMES, 85, seed=18, bit_depth=10),
]
SERVE_CLASSES = [
    _spec("s720_8", 1280, 720, CLASS_FRAMES, 60, seed=21),
    _spec("s720_10", 1280, 720, CLASS_FRAMES, 60, seed=22, bit_depth=10),
    _spec("s1080_8", 1920, 1080, CLASS_FRAMES, 60, seed=23),
    _spec("s1080_10", 1920, 1080, CLASS_FRAMES, 60, seed=24, bit_depth=10),
    _spec("s2160_8", 3840, 2160, CLASS_FRAMES, 60, seed=25),
    _spec("s2160_10", 3840, 2160, CLASS_FRAMES, 60, seed=26, bit_depth=10),
]


def cache_path(spec):
    digest = hashlib.sha1(json.dumps(spec, sort_keys=True).encode()).hexdigest()[:10]
    return os.path.join(STREAM_DIR, f"{spec['name']}-{digest}.ivf")


def cached(spec):
    """True when the stream's IVF is in the cache."""
    return os.path.exists(cache_path(spec))


def packets(spec, generate=True):
    """The stream's packets, from the cache; generated (and cached) first
    when missing, in a child process, unless generate is False (then
    FileNotFoundError)."""
    path = cache_path(spec)
    if not os.path.exists(path):
        if not generate:
            raise FileNotFoundError(path)
        ensure_cached([spec])
    with open(path, "rb") as f:
        return containers.ivf_packets(f.read())


def _generate(spec):
    """Generates the stream into the cache (in this process)."""
    path = cache_path(spec)
    if not os.path.exists(path):
        from . import streams  # the generator
        cfg = streams.config(spec["width"], spec["height"], spec["frames"], spec["q"], bit_depth=spec["bit_depth"],
                             chroma=spec["chroma"], tile_cols_log2=spec["tile_cols_log2"],
                             golden_interval=spec["golden_interval"], seed=spec["seed"], pan=spec["pan"],
                             rectangles=spec["rectangles"], noise=spec["noise"], color_space=spec["color_space"])
        pk = streams.generate(cfg)
        os.makedirs(STREAM_DIR, exist_ok=True)
        tmp = path + f".tmp{os.getpid()}"
        with open(tmp, "wb") as f:
            f.write(containers.ivf_write(pk, spec["width"], spec["height"]))
        os.replace(tmp, path)


def ensure_cached(specs, jobs=None):
    """Fills the cache for `specs` in child processes (the caller loads
    neither the generator nor its library): up to `jobs` of them at once
    (default: the host's cores), the largest streams dealt out first so the
    children finish together."""
    missing = [s for s in specs if not cached(s)]
    if not missing:
        return
    import subprocess
    import sys
    jobs = max(1, min(len(missing), jobs or os.cpu_count() or 1))
    work = sorted(missing, key=lambda s: -s["width"] * s["height"] * s["frames"])
    shares = [[] for _ in range(jobs)]
    load = [0] * jobs
    for s in work:
        k = load.index(min(load))
        shares[k].append(s)
        load[k] += s["width"] * s["height"] * s["frames"]
    code = ("import json, sys; sys.path.insert(0, sys.argv[1]); from rv9 import workloads; "
            "[workloads._generate(s) for s in json.loads(sys.argv[2])]")
    procs = [subprocess.Popen([sys.executable, "-c", code, os.path.dirname(_HERE), json.dumps(share)])
             for share in shares]
    codes = [p.wait() for p in procs]
    if any(codes):
        raise RuntimeError(f"stream generation failed (exit codes {codes})")


def looped(pk, n):
    """`pk` repeated to `n` packets (each repeat starts at the key frame, so
    the looped stream is a valid one)."""
    return [pk[i % len(pk)] for i in range(n)]


def luma_samples(spec):
    return spec["width"] * spec["height"]
