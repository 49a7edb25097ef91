"""Load the committed golden fixtures (tests/golden/*.npz) back into models."""
import hashlib
import os

import numpy as np

from ufem_b200 import meshgen as mg

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
STATIC_CASES = ["plate_64x16", "plate_6x3_distorted", "plate_4x2_strain", "plate_4x2_prescribed",
                "brick_3x2x2_distorted", "beam_20x5x5"]


def load(name):
    return np.load(os.path.join(GOLDEN, f"{name}.npz"), allow_pickle=False)


def model_from(z) -> mg.Model:
    def split(cnt, vals):
        out, o = [], 0
        for c in cnt:
            out.append(np.asarray(vals[o:o + c], np.float64))
            o += c
        return out
    m = mg.Model(n_xyz=z["m_xyz"], e_type=z["m_etype"], e_rs=z["m_ers"], e_mp=z["m_emp"],
                 e_nodes=z["m_enodes"], rs_type=z["m_rstype"], rs_vals=split(z["m_rscnt"], z["m_rsvals"]),
                 mp_type=z["m_mptype"], mp_vals=split(z["m_mpcnt"], z["m_mpvals"]),
                 nl_node=z["m_nlnode"], nl_type=z["m_nltype"], nl_dir=z["m_nldir"], nl_val=z["m_nlval"])
    if "mc_vars" in z.files:
        m.mc_vars = z["mc_vars"]
        m.mc_ilen = int(z["mc_ilen"])
        m.mc_olen = int(z["mc_olen"])
    return m


def model_sha(model: mg.Model) -> str:
    """One hash over every model table: a fixture that stores only results
    regenerates its model with the mesh generator and checks it with this."""
    rs_frm, rs_cnt, rs_vals = model.rs_flat()
    mp_frm, mp_cnt, mp_vals = model.mp_flat()
    tables = dict(m_xyz=model.n_xyz, m_etype=model.e_type, m_ers=model.e_rs, m_emp=model.e_mp,
                  m_enodes=model.e_nodes, m_rstype=model.rs_type, m_rscnt=rs_cnt, m_rsvals=rs_vals,
                  m_mptype=model.mp_type, m_mpcnt=mp_cnt, m_mpvals=mp_vals, m_nlnode=model.nl_node,
                  m_nltype=model.nl_type, m_nldir=model.nl_dir, m_nlval=model.nl_val)
    h = hashlib.sha256()
    for k, v in sorted(tables.items()):
        h.update(k.encode())
        h.update(np.ascontiguousarray(v).tobytes())
    return h.hexdigest()
