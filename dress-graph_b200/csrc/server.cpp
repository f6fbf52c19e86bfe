// server.cpp -- continuous-batching request loop (see dress_b200_ext.h).
#include "engine.h"
