"""Helpers shared by the GPU tests (device films through torch, hit mapping)."""
import numpy as np


def render_film(cr, scene, W, H, spp, seeds, estimator=0, max_bounce=7, window=None, wave_paths=0):
    """Accumulate renders with the given seeds into one device film and return
    an oracle.Film-like (sum, sumsq, count) view."""
    import torch
    import oracle
    x0, y0, x1, y1 = window or (0, 0, W, H)
    n = (x1 - x0) * (y1 - y0)
    s = torch.zeros(n * 3, dtype=torch.float64, device="cuda")
    q = torch.zeros(n * 3, dtype=torch.float64, device="cuda")
    c = torch.zeros(n, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for seed in seeds:
        d = cr.render_desc(W, H, spp, max_bounce=max_bounce, estimator=estimator, seed=seed, window=window,
                           wave_paths=wave_paths)
        scene.render_device(d, s.data_ptr(), q.data_ptr(), c.data_ptr(), stream=stream)
    torch.cuda.synchronize()
    shp = (y1 - y0, x1 - x0)
    return oracle.Film(s.cpu().numpy().reshape(*shp, 3), q.cpu().numpy().reshape(*shp, 3),
                       c.cpu().numpy().astype(np.uint32).reshape(shp))


def zscores(a, b):
    """|difference| over the combined standard error; a relative floor of 1e-6
    keeps pixels whose samples are all alike (a light seen directly) from
    turning float rounding into huge scores."""
    floor = (1e-6 * np.maximum(np.abs(a.mean), np.abs(b.mean))) ** 2
    return np.abs(a.mean - b.mean) / np.sqrt(a.var_of_mean + b.var_of_mean + floor + 1e-30)


def kind_index(prim, n_mesh):
    """(kind, index) from scene-order primitive ids: meshes first, then spheres."""
    prim = np.asarray(prim)
    kind = np.where(prim < 0, -1, np.where(prim < n_mesh, 0, 1))
    index = np.where(prim < 0, -1, np.where(prim < n_mesh, prim, prim - n_mesh))
    return kind, index
