/* OpenCV subset for the reference build (test infrastructure): see ../opencv_subset.h */
#include "../opencv_subset.h"
