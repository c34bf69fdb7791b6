/* utilsSource/intFloat/intFloat.h -- TEST INFRASTRUCTURE ONLY: empty stand-in
 * (nothing from it is used by Cullst/cullIslands.c). */
