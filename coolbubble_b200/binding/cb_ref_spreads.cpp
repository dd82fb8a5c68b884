/* cb_ref_spreads.cpp -- bubble.cpp with a setter for its spread sums.
 *
 * CoolBubble keeps the spreads that outEP prints (EtotVar ... avphiPVar) as
 * file-static variables of src/bubble.cpp (bubble.cpp:44), which code outside
 * that file cannot set. When the time loop runs on the GPU (cb_main_loop.hpp),
 * the spreads come from the library and must land in those variables before
 * outEP writes a line. A CoolBubble tree would add the one function below to
 * bubble.cpp; this translation unit does the same without editing the file:
 * it compiles bubble.cpp (its path in CBREF_BUBBLE_CPP) together with the
 * setter, and takes bubble.cpp's place in the link.
 */
#include CBREF_BUBBLE_CPP

void cb_ref_set_spreads(double etot_var, double ekin_var, double egrad_var, double epot_var, double avphi_var,
                        double avphip_var) {
    EtotVar = etot_var;
    EkintotVar = ekin_var;
    EgradtotVar = egrad_var;
    EpottotVar = epot_var;
    avphiVar = avphi_var;
    avphiPVar = avphip_var;
}
