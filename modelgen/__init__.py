"""Model builder for the tests and the benchmark (not part of the engine).

``modelgen.solver`` restates the reference's Python setup (rfnetwork/solver.py)
so that tests and ``bench.py`` can produce, on a machine where the reference
package cannot be imported, exactly the inputs its ``solve()`` hands the
engine; ``modelgen.configs`` builds the seeded workloads from it and
``modelgen.geometry`` holds the axis-aligned stand-ins for the pyvista shapes
the reference's setup reads. The engine product is ``rfnetwork_b200``.
"""
