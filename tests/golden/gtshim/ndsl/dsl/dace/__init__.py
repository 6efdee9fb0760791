from .orchestration import orchestrate  # noqa: F401
