"""Writes a patched copy of the reference's coupled-solver directory into oracle/_ref/patched/ (test infrastructure).

The patch is the reference-side binding of libdn_cuda that INTEGRATION.md §2 describes, applied by text
edits to copies of four files of src/core/coupled (all of that directory is copied, because its sources
include "solver.hpp" by relative path and every translation unit must see the same Solver layout):

  solver.hpp     + #include "dn_cuda.h", the lazily created handle `dn_` and its builder `dn()`
                   (defined in oracle/ref_cuda_binding.cpp);
  pressure.cpp   + a first branch in Solver::solve_pressure_correction (pressure.cpp:1031-1089) that hands
                   every `cuda_*` pressure_scheme to dn_pressure_solve;
  phase_field.cpp + a first branch in Solver::solve_phase_linear_system_eq25 (phase_field.cpp:437-503) that
                   hands ch_solver = cuda_sparse_pcg to dn_ch_linear_solve;
  operators.cpp  Solver::use_liu_pressure_split (operators.cpp:400-409) reads the scheme name without the
                   `cuda_` prefix, so that cuda_split_* keeps the split extrapolation and correction.

Nothing else of the reference changes.  oracle/Makefile (target refcuda) compiles the patched directory with
the unpatched src/core/base and src/core/linear_algebra headers, oracle/ref_harness.cpp (with
DN_REF_CUDA_BACKEND: the harness prefixes the schemes with `cuda_`) and oracle/ref_cuda_binding.cpp into
oracle/_ref/libdnref_cuda.so, linked against ding_nsch_core_solver_b200/libdn_cuda.so.

    DN_REFERENCE=<reference tree> python oracle/patch_reference.py
"""
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref", "patched", "src", "core", "coupled")


def edit(text, old, new, what):
    if text.count(old) != 1:
        raise SystemExit(f"patch_reference: anchor for {what} found {text.count(old)} times (expected 1)")
    return text.replace(old, new)


def patch_solver_hpp(t):
    t = edit(t, '#include "core/linear_algebra/ch_sparse_krylov.hpp"\n',
             '#include "core/linear_algebra/ch_sparse_krylov.hpp"\n#include "dn_cuda.h"\n', "solver.hpp include")
    # the handle and its builder, as the first private members
    idx = t.index("private:")
    t = t[:idx] + ("private:\n  mutable dn_handle *dn_ = nullptr;\n  dn_handle *dn() const;\n"
                   + t[idx + len("private:"):])
    return t


def patch_pressure_cpp(t):
    old = '  if (cfg_.pressure_scheme == "petsc_pcg") {\n    solver_name = "PETSc";'
    new = ('  if (cfg_.pressure_scheme.rfind("cuda_", 0) == 0) {\n'
           '    solver_name = "CUDA";\n'
           '    int its = 0;\n'
           '    double rel = 0.0;\n'
           '    const dn_status s = dn_pressure_solve(dn(), current_step_index_, u_star_.data.data(), '
           'v_star_.data.data(),\n'
           '                                          rho_mid_.data.data(), pressure_.data.data(),\n'
           '                                          pressure_previous_step_.data.data(), '
           'pressure_correction_.data.data(),\n'
           '                                          &its, &rel);\n'
           '    if (s != DN_OK) throw std::runtime_error(dn_last_error(dn_));\n'
           '    last_pressure_iterations_ = its;\n'
           '    residual = rel;\n'
           '  } else if (cfg_.pressure_scheme == "petsc_pcg") {\n    solver_name = "PETSc";')
    return edit(t, old, new, "pressure dispatcher")


def patch_phase_field_cpp(t):
    old = ('  (void)target_mean;\n  if (cfg_.ch_solver == "petsc_pcg") {\n')
    new = ('  (void)target_mean;\n'
           '  if (cfg_.ch_solver == "cuda_sparse_pcg") {\n'
           '    int its = 0;\n'
           '    const dn_status s = dn_ch_linear_solve(dn(), rhs_field.data.data(), alpha0, c_state.data.data(),\n'
           '                                           &iterate_residual, &equation_residual, &its);\n'
           '    if (s != DN_OK) throw std::runtime_error(dn_last_error(dn_));\n'
           '    last_ch_iterations_ = its;\n'
           '    last_ch_solver_name_ = "CUDA[SparsePCG]";\n'
           '    return;\n'
           '  }\n'
           '  if (cfg_.ch_solver == "petsc_pcg") {\n')
    return edit(t, old, new, "CH dispatcher")


def patch_operators_cpp(t):
    head = "bool Solver::use_liu_pressure_split() const {\n"
    start = t.index(head)
    end = t.index("}\n", start)
    body = t[start + len(head):end]
    body = body.replace("cfg_.pressure_scheme ==", "scheme ==")
    body = ('  const std::string scheme = cfg_.pressure_scheme.rfind("cuda_", 0) == 0 ? cfg_.pressure_scheme.substr(5)\n'
            '                                                                       : cfg_.pressure_scheme;\n'
            + body)
    return t[:start + len(head)] + body + t[end:]


def main():
    ref = os.environ.get("DN_REFERENCE")
    if not ref or not os.path.isdir(ref):
        raise SystemExit("set DN_REFERENCE to the reference tree")
    src = os.path.join(ref, "src", "core", "coupled")
    if os.path.isdir(OUT):
        shutil.rmtree(OUT)
    os.makedirs(OUT)
    for name in sorted(os.listdir(src)):
        if name.endswith((".cpp", ".hpp")):
            shutil.copyfile(os.path.join(src, name), os.path.join(OUT, name))
    for name, fn in (("solver.hpp", patch_solver_hpp), ("pressure.cpp", patch_pressure_cpp),
                     ("phase_field.cpp", patch_phase_field_cpp), ("operators.cpp", patch_operators_cpp)):
        path = os.path.join(OUT, name)
        with open(path) as f:
            text = f.read()
        with open(path, "w") as f:
            f.write(fn(text))
    print(f"patched copy written to {OUT}", file=sys.stderr)


if __name__ == "__main__":
    main()
