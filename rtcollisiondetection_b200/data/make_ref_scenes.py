"""Generate ``ref_scenes.npz``: the reference's benchmark shelf scenes.

A data-preparation script, run once where the upstream model files are
available.  It reads the OBJ models of ``models/curobo`` and stores each one
deduplicated the way the upstream loader does it (a vertex is identified by
its exact float position, first occurrence wins, faces in file order,
``RTCD/Meshes/mesh.h:218-231``; polygons fan-triangulated), plus the three
scenes' compositions: which models, translated by how much
(``RTCD/CollisionScenes/Scene/shelfSimple.h``, ``shelf.h``, ``denseShelf.h``:
every obstacle is an identity pose translated by a vector, scale 1, applied
to the vertices in float as ``meshModel(path, pose, scale)`` does,
``RTCD/Meshes/mesh.h:258-270``).

Usage:  python make_ref_scenes.py <models/curobo dir> <out.npz>
"""
import os
import sys

import numpy as np

from make_panda import dedupe_mesh, parse_obj

# (model, translation) per scene, in the order the scene headers add them
SCENES = {
    'simple': [('shelves', (0.45, 0.0, 0.4)), ('bin', (0.0, -0.6, 0.0)), ('bin', (0.0, 0.6, 0.0))],
    'medium': [('shelves', (0.45, 0.0, 0.4)), ('bin', (0.0, -0.6, 0.0)), ('bin', (0.0, 0.6, 0.0)),
               ('Bob', (-0.4, 0.0, 0.0)), ('Cow', (-0.4, 0.0, 0.0)), ('Fish', (-0.4, 0.0, 0.0)),
               ('Sheep', (-0.4, 0.0, 0.0)), ('Snakeboard', (-0.4, 0.0, 0.0))],
    'dense': [('shelves', (0.45, 0.0, 0.4)), ('bin_dense', (0.0, -0.6, 0.0)), ('bin_dense', (0.0, 0.6, 0.0)),
              ('Bob', (-0.4, 0.0, 0.0)), ('Face1', (-0.4, 0.0, 0.0)), ('Face2', (-0.4, 0.0, 0.0)),
              ('Face3', (-0.4, 0.0, 0.0)), ('Cow', (-0.4, 0.0, 0.0)), ('Fish', (-0.4, 0.0, 0.0)),
              ('Sheep', (-0.4, 0.0, 0.0)), ('Snakeboard', (-0.4, 0.0, 0.0))],
}


def main(src, out):
    arrays = {}
    models = sorted({m for parts in SCENES.values() for m, _ in parts})
    for m in models:
        raw, faces = parse_obj(os.path.join(src, m + '.obj'))
        v, t, _ = dedupe_mesh(raw, faces)
        arrays['model_%s_verts' % m] = v
        arrays['model_%s_tris' % m] = t
        print(m, len(v), 'verts', len(t), 'tris')
    for name, parts in SCENES.items():
        arrays['scene_%s_models' % name] = np.array([m for m, _ in parts])
        arrays['scene_%s_offsets' % name] = np.array([o for _, o in parts], np.float32)
        print(name, sum(len(arrays['model_%s_tris' % m]) for m, _ in parts), 'tris')
    np.savez_compressed(out, **arrays)


if __name__ == '__main__':
    main(sys.argv[1], sys.argv[2])
