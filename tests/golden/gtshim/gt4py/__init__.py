"""Stand-in for gt4py (absent here): only what pySHiELD's stencils import."""
