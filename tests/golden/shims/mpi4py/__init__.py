"""Single-rank stand-in for mpi4py, used only to import the reference tracker
in this container when generating golden vectors (mpi4py is not installed)."""
