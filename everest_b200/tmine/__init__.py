"""Query driver with the reference's ``tmine`` surface (system/tmine/): YAML
queries (``Query``), ``frontend.Mining`` / ``MiningSingle`` and the
``@@@ [output starts]`` / ``@@@ [output ends]`` CLI output, over the
``corelib`` module of this package."""
