/* oracle shim: nothing to declare */
