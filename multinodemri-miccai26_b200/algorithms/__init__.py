"""TVM / TVME / TVMW reconstructors and CLI mains on the b200 backend."""
