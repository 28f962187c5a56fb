"""Generate tests/golden/replay_bvh2.npz from the reference's own Python replay.

Runs in the development container only (it imports tools/sunrt/replay_geometry.py from the
reference checkout given by --reference). The scenes are packed by the oracle's restated legacy
writers (median BVH2 leaves of four triangles, BVH2 top level, reflection_software.rs:170-264,
instance_bvh.rs:414-460) and every coordinate, transform and ray component is a small dyadic
rational, so every product and sum in the replay is exact and the only roundings are the
correctly rounded divisions and single multiplies that the oracle performs identically. The
replay's float32 results (t bits, hit record, traversal counters) are stored as golden vectors.

    python tests/golden/make_replay_golden.py --reference /path/to/renderlab

With --general it writes tests/golden/replay_bvh2_general.npz instead: general f32 inputs (jittered
height fields and triangle soups at arbitrary coordinates, instances under arbitrary rotations and
scales with f32 rows, rays aimed at triangle interiors, edges and vertices). There every product and
sum rounds. The replay forms its dot products with np.dot, whose summation order and fusing belong
to the host's BLAS library, so each case is traced twice: as the tool ships ("numpy"), and with
the replay's np.dot evaluated left to right in f32, one rounding a product and a sum
("sequential": the order the WGSL writes its dot products in and the oracle evaluates them). The
tool's own code is not changed; only the dot function it calls is swapped, through a stand-in for
its module's numpy. The test requires the sequential replay bit for bit and bounds the numpy one.
"""
from __future__ import annotations

import argparse
import json
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import oracle as O  # noqa: E402

REPLAY_COUNTERS = ('tlas_nodes', 'tlas_box_tests', 'tlas_instance_entries', 'instance_box_tests',
                   'instance_box_entries', 'blas_visits', 'blas_nodes', 'blas_box_tests',
                   'triangle_tests')


def dyadic_mesh(rng, nx, nz, step=0.25):
    """A height field of quads on a dyadic grid (heights in quarters)."""
    p = []
    for z in range(nz + 1):
        for x in range(nx + 1):
            p.append([x * step, float(rng.integers(0, 4)) * 0.25, z * step])
    i = []
    for z in range(nz):
        for x in range(nx):
            a = z * (nx + 1) + x
            b, c = a + 1, a + nx + 1
            i += [a, c, b, b, c, c + 1]
    return np.array(p, np.float32), np.array(i, np.uint32)


def instances(rng, n, meshes):
    model = np.zeros((n, 3, 4), np.float32)
    rows = np.zeros((n, 3, 4), np.float32)
    mesh = np.zeros(n, np.uint32)
    aux = np.zeros((n, 2), np.uint32)
    for k in range(n):
        s = float(2.0 ** int(rng.integers(-1, 2)))
        t = rng.integers(-16, 16, 3) * 0.5
        model[k, :, :3] = np.eye(3) * s
        model[k, :, 3] = t
        rows[k, :, :3] = np.eye(3) / s
        rows[k, :, 3] = -t / s
        mesh[k] = k % meshes
        aux[k] = (100 + k, 0 if k % 7 == 3 else 1)
    return dict(model=model, rows=rows, mesh=mesh, aux=aux)


def dyadic_rays(rng, n, lo, hi, inst):
    """Rays from dyadic origins toward dyadic points near random instances (most of them hit)."""
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3] = rng.integers(int(lo * 8), int(hi * 8), (n, 3)) / 8.0
    r[:, 1] = rng.integers(40, 80, n) / 8.0
    k = rng.integers(0, len(inst['mesh']), n)
    target = inst['model'][k, :, 3] + inst['model'][k, 0, 0][:, None] * (
        rng.integers(0, 6, (n, 3)) * 0.25)
    target[:, 1] = rng.integers(0, 4, n) * 0.25
    r[:, 4:7] = target - r[:, 0:3]
    miss = rng.random(n) < 0.2
    r[miss, 4:7] = rng.integers(-4, 5, (miss.sum(), 3)).astype(np.float32)
    # A few axis-aligned and zero-component directions exercise the 1e-30 inverse guard.
    r[::17, 4] = 0.0
    r[::23, 6] = 0.0
    r[:, 3] = rng.choice([0.0, 0.125], n)
    r[:, 7] = rng.choice([1e6, 4.0], n)
    return r


def general_mesh(rng, kind):
    """A height field with jittered, non-dyadic vertices, or a soup of 60 random triangles."""
    if kind == 0:
        nx, nz = 7, 6
        p = []
        for z in range(nz + 1):
            for x in range(nx + 1):
                p.append([x * 0.37 + rng.uniform(-0.1, 0.1), rng.uniform(-0.3, 0.3), z * 0.41 + rng.uniform(-0.1, 0.1)])
        i = []
        for z in range(nz):
            for x in range(nx):
                a = z * (nx + 1) + x
                b, c = a + 1, a + nx + 1
                i += [a, c, b, b, c, c + 1]
        return np.array(p, np.float32), np.array(i, np.uint32)
    centre = rng.uniform(-1.0, 1.0, 3)
    a = centre + rng.uniform(-1.3, 1.3, (60, 3))
    tri = np.concatenate([a, a + rng.normal(0, 0.4, (60, 3)), a + rng.normal(0, 0.4, (60, 3))], axis=1)
    return tri.reshape(-1, 3).astype(np.float32), np.arange(180, dtype=np.uint32)


def general_instances(rng, n, meshes):
    """Instances under uniformly random rotations, scales in [0.6, 1.7] and translations in a
    10-unit box; rows are the f64 inverse rounded to f32 (the caller supplies them, as the
    renderer does)."""
    model = np.zeros((n, 3, 4), np.float32)
    rows = np.zeros((n, 3, 4), np.float32)
    mesh = np.zeros(n, np.uint32)
    aux = np.zeros((n, 2), np.uint32)
    for k in range(n):
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        w, x, y, z = q
        rot = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                        [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                        [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])
        m = np.eye(4)
        m[:3, :3] = rot * rng.uniform(0.6, 1.7)
        m[:3, 3] = rng.uniform(-5.0, 5.0, 3)
        model[k] = m[:3].astype(np.float32)
        rows[k] = np.linalg.inv(model[k].astype(np.float64).tolist() + [[0, 0, 0, 1]])[:3].astype(np.float32)
        mesh[k] = k % meshes
        aux[k] = (200 + k, 0 if k % 5 == 2 else 1)
    return dict(model=model, rows=rows, mesh=mesh, aux=aux)


def general_rays(rng, n, meshes, inst):
    """Rays from random origins toward points of random instanced triangles: a third at interior
    points, a third at edge points, a sixth at vertices, a sixth past the triangle (misses)."""
    r = np.zeros((n, 8), np.float32)
    o = rng.uniform(-9.0, 9.0, (n, 3))
    o[:, 1] = rng.uniform(6.0, 12.0, n)
    k = rng.integers(0, len(inst['mesh']), n)
    target = np.zeros((n, 3))
    for j in range(n):
        p, i = meshes[int(inst['mesh'][k[j]])]
        t = int(rng.integers(0, len(i) // 3))
        v = p[i[3 * t:3 * t + 3]].astype(np.float64)
        c = j % 6
        if c < 2:
            w = rng.dirichlet([1, 1, 1])
        elif c < 4:
            e = rng.uniform()
            w = np.roll([e, 1 - e, 0.0], int(rng.integers(0, 3)))
        elif c == 4:
            w = np.roll([1.0, 0.0, 0.0], int(rng.integers(0, 3)))
        else:
            w = np.array([1.4, -0.2, -0.2])
        local = w @ v
        target[j] = inst['model'][k[j]].astype(np.float64) @ np.append(local, 1.0)
    r[:, 0:3] = o
    r[:, 4:7] = target - o
    r[:, 3] = rng.choice([0.0, 1e-3], n)
    r[:, 7] = rng.choice([1e6, 40.0], n)
    return r


class SequentialDot:
    """numpy, except that dot(a, b) of 1-D float32 vectors sums a[i] * b[i] left to right in f32."""

    def __getattr__(self, name):
        return getattr(np, name)

    @staticmethod
    def dot(a, b):
        a, b = np.asarray(a), np.asarray(b)
        if a.ndim != 1 or b.ndim != 1 or a.dtype != np.float32 or b.dtype != np.float32:
            return np.dot(a, b)
        acc = np.float32(a[0] * b[0])
        for k in range(1, len(a)):
            acc = np.float32(acc + np.float32(a[k] * b[k]))
        return acc


def write_geometry(directory: Path, words: np.ndarray, n_inst: int, top: bool, meshes_meta):
    path = directory / 'scene.json'
    words.astype('<u4').tofile(path.with_suffix('.words.bin'))
    path.write_text(json.dumps(dict(
        version=1, format='reflection-bvh2-u32-le', path='nonrt-software-reflections',
        hardware_acceleration_structures=False, header_words=8, instance_words=24,
        payload_words=int(len(words)), frame=1, view=0, generation=1,
        written_instances=int(words[0]), reserved_instances=n_inst,
        tlas=dict(base_word=int(words[1]), root=int(words[2]), refits=int(words[3])),
        source_draws=[dict(placements=[dict(included=True)] * int(words[0]))],
        meshes=meshes_meta)))
    return path


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--reference', required=True, type=Path)
    ap.add_argument('--out', type=Path, default=Path(__file__).with_name('replay_bvh2.npz'))
    ap.add_argument('--general', action='store_true', help='general f32 inputs (replay_bvh2_general.npz)')
    args = ap.parse_args()
    sys.path.insert(0, str(args.reference / 'tools' / 'sunrt'))
    import replay_geometry
    from replay_geometry import Geometry  # the reference's own replay

    rng = np.random.default_rng(0x5EED if not args.general else 0x6E4E)
    if args.general and args.out.name == 'replay_bvh2.npz':
        args.out = args.out.with_name('replay_bvh2_general.npz')
    cases = {}
    for name, n_inst, tlas_mode in (('flat', 6, 0), ('tlas', 48, 1)):
        if args.general:
            meshes = [general_mesh(rng, 0), general_mesh(rng, 1)]
            inst = general_instances(rng, n_inst, len(meshes))
        else:
            meshes = [dyadic_mesh(rng, 6, 5), dyadic_mesh(rng, 4, 4)]
            inst = instances(rng, n_inst, len(meshes))
        words = O.scene_words(O.KIND_RS_BVH2, meshes, inst, tlas_mode=tlas_mode)
        rays = general_rays(rng, 600, meshes, inst) if args.general else dyadic_rays(rng, 400, -8.0, 12.0, inst)
        with tempfile.TemporaryDirectory() as d:
            geo = Geometry(write_geometry(Path(d), words, n_inst, tlas_mode == 1, []))
            t = np.zeros(len(rays), np.uint32)
            rec = np.zeros((len(rays), 4), np.uint32)
            cnt = np.zeros((len(rays), len(REPLAY_COUNTERS)), np.uint64)
            for dot in (('numpy', 'sequential') if args.general else ('numpy',)):
                replay_geometry.np = SequentialDot() if dot == 'sequential' else np
                for any_hit in (False, True):
                    for k, r in enumerate(rays):
                        res = geo.trace(r[0:3], r[4:7], r[3], r[7], any_hit)
                        t[k] = np.float32(res['t']).view(np.uint32)
                        rec[k] = res['record']
                        cnt[k] = [res[c] for c in REPLAY_COUNTERS]
                    key = f'{name}_{"any" if any_hit else "closest"}' + (f'_{dot}' if args.general else '')
                    cases[key + '_t'] = t.copy()
                    cases[key + '_record'] = rec.copy()
                    cases[key + '_counters'] = cnt.copy()
            replay_geometry.np = np
            del geo.f
            geo.w._mmap.close()
        cases[name + '_words'] = words
        cases[name + '_rays'] = rays
    np.savez_compressed(args.out, counters=np.array(REPLAY_COUNTERS), **cases)
    print(f'wrote {args.out} ({args.out.stat().st_size} bytes)')


if __name__ == '__main__':
    main()
