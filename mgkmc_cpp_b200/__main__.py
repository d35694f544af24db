"""Command line of the package, in place of the reference executable:

    python -m mgkmc_cpp_b200 [config.yaml]

reads the reference's YAML keys (default cpp_config.yaml, as main.cpp:27) and
runs simulation_type "kmc" or "linear_elastic" on the GPU, writing the same
logs and VTU files into output.directory."""
import sys

from . import run_config


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    path = argv[0] if argv else "cpp_config.yaml"
    run_config(path)
    return 0


if __name__ == "__main__":
    sys.exit(main())
