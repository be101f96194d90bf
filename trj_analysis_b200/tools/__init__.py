"""Command-line tools with the call shapes of the reference programs for this path."""
