"""unidock_tools: Python side of the B200 docking engine (binding over the C ABI,
synthetic inputs, torch autograd of the fixed-pose energy)."""
