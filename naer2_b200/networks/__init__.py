"""Network builders of the benchmark configurations, written in the DSL."""
