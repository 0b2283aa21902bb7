"""GPU solvers behind the reference's solver interfaces."""
