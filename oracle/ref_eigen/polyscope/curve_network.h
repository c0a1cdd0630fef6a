#pragma once
#include "polyscope.h"
