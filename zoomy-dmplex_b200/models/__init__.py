"""Generated SME model plugins (Model.H / Numerics.H per directory) and
their generator (gen_sme.py).  ``parameter_table`` reads a model's parameter
names and defaults from its generated header."""
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))


def available():
    return sorted(d for d in os.listdir(HERE) if os.path.exists(os.path.join(HERE, d, "Model.H")))


def header_path(model: str, which: str = "Model.H") -> str:
    return os.path.join(HERE, model, which)


def parameter_table(model: str):
    with open(header_path(model)) as f:
        src = f.read()
    names = re.search(r"parameter_names\(\) \{ return \{ (.*?) \}; \}", src).group(1)
    vals = re.search(r"default_parameters\(\) \{ return \{ (.*?) \}; \}", src).group(1)
    names = [s.strip().strip('"') for s in names.split(",")]
    vals = [float(v) for v in vals.split(",")]
    return names, vals


def constants(model: str):
    with open(header_path(model)) as f:
        src = f.read()
    out = {}
    for k in ("n_dof_q", "n_dof_qaux", "n_parameters", "dimension"):
        out[k] = int(re.search(r"static constexpr int %s\s*=\s*(\d+);" % k, src).group(1))
    return out


def boundary_tags(model: str):
    """The model's boundary tag names (Model::get_boundary_tags), in bc-index order."""
    with open(header_path(model)) as f:
        src = f.read()
    body = re.search(r"get_boundary_tags\(\) \{ return \{ (.*?) \}; \}", src).group(1)
    return [t.strip().strip('"') for t in body.split(",")]
