/* Case-sensitive alias: the reference includes both <windows.h> and <Windows.h>. */
#pragma once
#include "windows.h"
