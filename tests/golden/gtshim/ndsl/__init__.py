"""Stand-in for NDSL (absent here): the names pySHiELD imports, nothing more."""
