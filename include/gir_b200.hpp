#pragma once
#include "gir_dev.h"
