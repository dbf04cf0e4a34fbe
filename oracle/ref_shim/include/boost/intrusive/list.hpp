/* oracle shim (test infrastructure only): the reference includes this header but uses nothing from it on the engine path */
