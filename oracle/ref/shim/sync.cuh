/* empty stand-in (oracle/_ref build only) */
