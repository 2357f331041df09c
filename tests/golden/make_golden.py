"""Generate tests/golden/cuba_reference.json from the reference tree.

Sources (Brian 1.4.4 tree, read at generation time only):
  dev/benchmarking/cuba/CUBA.cpp:47-53 .......... propagator constants of the
      CUBA model (taum 20, taue 5, taui 10 ms, dt 0.1 ms), as the reference's
      hand-written C++ benchmark hard-codes them (8 significant digits, the
      matrix transposed, C in mV)
  dev/benchmarking/cuba/data/cpp_cuba_results.py  per-run spike counts of the
      C++ CUBA benchmark (2.5 s, refractory 5 ms, 80 synapses per neuron)
  dev/benchmarking/cuba/data/brian_cuba_results_compile_nounits.pkl
      per-run spike counts of Brian itself on the same benchmark

Run: python tests/golden/make_golden.py [reference_root]
"""
import json
import os
import pickle
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(root):
    cuba = os.path.join(root, "dev", "benchmarking", "cuba")
    src = open(os.path.join(cuba, "CUBA.cpp"), encoding="latin1").read()
    amat = re.search(r"Amatvals\[3\]\[3\]\s*=\s*\{(.*?)\};", src, re.S).group(1)
    rows = re.findall(r"\{([^}]*)\}", amat)
    A_t = [[float(x) for x in r.split(",")] for r in rows]
    cvec = re.search(r"Cvecvals\[3\]\s*=\s*\{([^}]*)\}", src).group(1)
    C_mV = [float(x) for x in cvec.split(",")]
    ns = {}
    exec(open(os.path.join(cuba, "data", "cpp_cuba_results.py")).read(), ns)
    cpp = {str(n): [c for _, c in runs] for (n, _, _, runs) in ns["cpp_cuba"]}
    with open(os.path.join(cuba, "data", "brian_cuba_results_compile_nounits.pkl"), "rb") as f:
        br = pickle.load(f, encoding="latin1")
    brian = {str(int(n)): [int(c) for _, c in runs] for (n, _, _, runs) in br}
    out = {
        "cuba_propagator": {"A_transposed": A_t, "C_mV": C_mV, "significant_digits": 8,
                            "source": "dev/benchmarking/cuba/CUBA.cpp:47-53"},
        "cuba_benchmark_spike_counts": {
            "setup": "N neurons (80% exc), p = 80/N, we = 1.62 mV, wi = -9 mV, refractory 5 ms, 2.5 s, dt 0.1 ms",
            "cpp": cpp, "brian_compile_nounits": brian,
            "source": "dev/benchmarking/cuba/data/cpp_cuba_results.py, brian_cuba_results_compile_nounits.pkl"},
    }
    with open(os.path.join(HERE, "cuba_reference.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("BRIAN_REFERENCE", "/root/reference"))
