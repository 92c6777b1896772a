"""Small helpers shared by the tests."""
import hashlib
import re

import numpy as np


def sha(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def parse_cfg(text: str) -> dict:
    """key=value lines with # comments, as the reference's load_config reads them."""
    out = {}
    for line in text.splitlines():
        line = line.split("#", 1)[0]
        if "=" not in line:
            continue
        k, v = line.split("=", 1)
        out[k.strip()] = v.strip()
    return out


def cfg_params(text: str) -> dict:
    """The reference Config fields the path uses, with the reference's defaults."""
    c = parse_cfg(text)
    l0 = float(c.get("l0", 0.01))
    re_ratio = float(c.get("re_ratio", 2.1))
    return {
        "l0": l0,
        "re": re_ratio * l0,  # the product run_benchmark passes (src/lsmps.cpp:73)
        "max_neighbors": int(c.get("max_neighbors", 96)),
        "wls_samples": int(c.get("wls_samples", 4096)),
        "ppe_max_unknowns": int(c.get("ppe_max_unknowns", 12000)),
        "ppe_max_iter": int(c.get("ppe_max_iter", 400)),
        "ppe_tol": float(c.get("ppe_tol", 1e-9)),
    }


TIMING_FIELDS = re.compile(r'("(?:assembly_ms|solve_ms)": )[-0-9.e+]+')


def strip_json_timings(text: str) -> str:
    return TIMING_FIELDS.sub(r"\1<t>", text)


def strip_csv_timings(text: str) -> str:
    lines = text.splitlines()
    head, row = lines[0], lines[1].split(",")
    return head + "\n" + ",".join(row[:-2])


def jittered_lattice(nx, jitter=0.1, seed=0, l0=1.0):
    rng = np.random.default_rng(seed)
    g = np.stack(np.meshgrid(np.arange(nx), np.arange(nx), np.arange(nx), indexing="ij"), -1).reshape(-1, 3)
    g = g[:, ::-1].astype(np.float64)
    return ((g + 0.5 + rng.uniform(-jitter, jitter, g.shape)) * l0).astype(np.float64)
