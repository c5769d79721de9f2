"""Python FFI wrappers over the TorchScript classes, in the style of hastypy.ffi."""
