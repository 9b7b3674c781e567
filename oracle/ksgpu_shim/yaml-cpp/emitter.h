// Minimal stand-in for yaml-cpp's emitter.h (oracle/_ref build only).
#include "yaml.h"
