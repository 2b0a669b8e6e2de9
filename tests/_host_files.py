"""Input files in the reference's formats, for tests of the host side."""
from lbx import host


def write_params(path, values):
    """A params.in in the positional layout: 'label value' per line."""
    with open(path, "w") as fh:
        for (name, is_real) in host.params_layout():
            v = values.get(name, 0.0 if is_real else 0)
            label = name.replace("[", "_").replace("]", "")
            fh.write("%-24s %s\n" % (label, repr(float(v)) if is_real else str(int(v))))
