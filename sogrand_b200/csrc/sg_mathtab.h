/* Generated by gen_mathtab.py -- do not edit.  Constants and tables of
 * the decoder's own exp/log (see sg_math.h).  All values are round-to-
 * nearest binary64 images of exact quantities computed with mpmath. */
#pragma once
#define SG_EXP_INV_LN2_N 0x1.71547652b82fep+7  /* N/ln2, N = 128 */
#define SG_EXP_LN2_N_HI 0x1.62e42fef80000p-8  /* ln2/N, 35 significant bits */
#define SG_EXP_LN2_N_LO 0x1.1cf79abc9e3b4p-43  /* ln2/N - SG_EXP_LN2_N_HI */
#define SG_EXP_SHIFT 0x1.8p52
#define SG_EXP_C2 0x1.0000000000000p-1  /* 1/2! */
#define SG_EXP_C3 0x1.5555555555555p-3  /* 1/3! */
#define SG_EXP_C4 0x1.5555555555555p-5  /* 1/4! */
#define SG_EXP_C5 0x1.1111111111111p-7  /* 1/5! */
#define SG_EXP_C6 0x1.6c16c16c16c17p-10  /* 1/6! */
#define SG_EXP_C7 0x1.a01a01a01a01ap-13  /* 1/7! */
/* {H_j, t_j}: 2^(j/128) ~= H_j * (1 + t_j) */
#define SG_EXP_TAB_INIT { \
  0x1.0000000000000p+0, 0x0.0p+0, \
  0x1.0163da9fb3335p+0, 0x1.b3b4f1a88bf6ep-54, \
  0x1.02c9a3e778061p+0, -0x1.160139cd8dc5dp-56, \
  0x1.04315e86e7f85p+0, -0x1.05e7a108766d1p-54, \
  0x1.059b0d3158574p+0, 0x1.cd2523567f613p-55, \
  0x1.0706b29ddf6dep+0, -0x1.bce8023f98efap-55, \
  0x1.0874518759bc8p+0, 0x1.0f74e61e6c861p-57, \
  0x1.09e3ecac6f383p+0, 0x1.0a3e45b33d399p-54, \
  0x1.0b5586cf9890fp+0, 0x1.79aa65d837b6dp-54, \
  0x1.0cc922b7247f7p+0, 0x1.eb51a92fdeffcp-55, \
  0x1.0e3ec32d3d1a2p+0, 0x1.ebe3d702f9cd1p-60, \
  0x1.0fb66affed31bp+0, -0x1.a033489906e0bp-57, \
  0x1.11301d0125b51p+0, -0x1.556522a2fbd0ep-54, \
  0x1.12abdc06c31ccp+0, -0x1.080ef8c4eea55p-58, \
  0x1.1429aaea92de0p+0, -0x1.1c923b9d5f416p-54, \
  0x1.15a98c8a58e51p+0, 0x1.0d3e3e95c55afp-55, \
  0x1.172b83c7d517bp+0, -0x1.01b15eaa59348p-55, \
  0x1.18af9388c8deap+0, -0x1.f1ff055de323dp-55, \
  0x1.1a35beb6fcb75p+0, 0x1.b898c3f1353bfp-55, \
  0x1.1bbe084045cd4p+0, -0x1.6d99c7611eb26p-54, \
  0x1.1d4873168b9aap+0, 0x1.aecf73e3a2f60p-54, \
  0x1.1ed5022fcd91dp+0, -0x1.fe782cb86389dp-55, \
  0x1.2063b88628cd6p+0, 0x1.a6f4144a6c38dp-55, \
  0x1.21f49917ddc96p+0, 0x1.07a05b0e4047dp-55, \
  0x1.2387a6e756238p+0, 0x1.68efde3a8a894p-54, \
  0x1.251ce4fb2a63fp+0, 0x1.75e18f274487dp-55, \
  0x1.26b4565e27cddp+0, 0x1.0472b981fe7f2p-55, \
  0x1.284dfe1f56381p+0, -0x1.6b87b3f71085ep-54, \
  0x1.29e9df51fdee1p+0, 0x1.2f7e16d09ab31p-55, \
  0x1.2b87fd0dad990p+0, -0x1.d219b1a6fbffap-60, \
  0x1.2d285a6e4030bp+0, 0x1.b3782720c0ab4p-55, \
  0x1.2ecafa93e2f56p+0, 0x1.e149289cecb8fp-57, \
  0x1.306fe0a31b715p+0, 0x1.34d754db0abb6p-55, \
  0x1.32170fc4cd831p+0, 0x1.64201e2ac744cp-55, \
  0x1.33c08b26416ffp+0, 0x1.fdd395dd3f84ap-55, \
  0x1.356c55f929ff1p+0, -0x1.6a3803b8e5b04p-55, \
  0x1.371a7373aa9cbp+0, -0x1.24aedcc4b5068p-54, \
  0x1.38cae6d05d866p+0, -0x1.907f81b512d8ep-54, \
  0x1.3a7db34e59ff7p+0, -0x1.1d1e83e9436d2p-56, \
  0x1.3c32dc313a8e5p+0, -0x1.91919b3ce1b15p-54, \
  0x1.3dea64c123422p+0, 0x1.59f48a72a4c6dp-55, \
  0x1.3fa4504ac801cp+0, -0x1.312607a28698ap-54, \
  0x1.4160a21f72e2ap+0, -0x1.8a78f4817895bp-58, \
  0x1.431f5d950a897p+0, -0x1.c2c9b67499a1bp-56, \
  0x1.44e086061892dp+0, 0x1.363ed60c2ac11p-59, \
  0x1.46a41ed1d0057p+0, 0x1.666093b0664efp-54, \
  0x1.486a2b5c13cd0p+0, 0x1.ecce1daa10379p-57, \
  0x1.4a32af0d7d3dep+0, 0x1.3ff8e3f0f1230p-54, \
  0x1.4bfdad5362a27p+0, 0x1.690cebb7aafb0p-56, \
  0x1.4dcb299fddd0dp+0, 0x1.31dbdeb54e077p-54, \
  0x1.4f9b2769d2ca7p+0, -0x1.f94340071a38ep-55, \
  0x1.516daa2cf6642p+0, -0x1.7deccdc93a349p-55, \
  0x1.5342b569d4f82p+0, -0x1.8dec6bd0f385fp-56, \
  0x1.551a4ca5d920fp+0, -0x1.61246ec7b5cf6p-55, \
  0x1.56f4736b527dap+0, 0x1.3350518fdd78ep-54, \
  0x1.58d12d497c7fdp+0, 0x1.b98b72f8a9b05p-56, \
  0x1.5ab07dd485429p+0, 0x1.063e1e21c5409p-54, \
  0x1.5c9268a5946b7p+0, 0x1.4c7855019c6eap-60, \
  0x1.5e76f15ad2148p+0, 0x1.432e62b64c035p-54, \
  0x1.605e1b976dc09p+0, -0x1.ce44a6199769fp-55, \
  0x1.6247eb03a5585p+0, -0x1.c33c53bef4da8p-55, \
  0x1.6434634ccc320p+0, -0x1.45378892be9aep-55, \
  0x1.6623882552225p+0, -0x1.3cedd78565858p-54, \
  0x1.68155d44ca973p+0, 0x1.710aa807e1964p-58, \
  0x1.6a09e667f3bcdp+0, -0x1.3b3efbf5e2228p-54, \
  0x1.6c012750bdabfp+0, -0x1.a12ad8734b982p-57, \
  0x1.6dfb23c651a2fp+0, -0x1.367efb86da9eep-57, \
  0x1.6ff7df9519484p+0, -0x1.0dc3d54e08851p-55, \
  0x1.71f75e8ec5f74p+0, -0x1.81f647e5a3ecfp-56, \
  0x1.73f9a48a58174p+0, -0x1.6ee4ac08b7db0p-55, \
  0x1.75feb564267c9p+0, -0x1.619321e55e68ap-55, \
  0x1.780694fde5d3fp+0, 0x1.09ccb5e09d4d3p-54, \
  0x1.7a11473eb0187p+0, -0x1.b32dcb94da51dp-56, \
  0x1.7c1ed0130c132p+0, 0x1.4ecfd5467c06bp-54, \
  0x1.7e2f336cf4e62p+0, 0x1.5ebe1abd66c55p-57, \
  0x1.80427543e1a12p+0, -0x1.8a1c52fb3cf42p-55, \
  0x1.82589994cce13p+0, -0x1.369b6f13b3734p-54, \
  0x1.8471a4623c7adp+0, -0x1.05e843a19ff1ep-55, \
  0x1.868d99b4492edp+0, -0x1.4d450d872576ep-54, \
  0x1.88ac7d98a6699p+0, 0x1.0ad675b0e8a00p-54, \
  0x1.8ace5422aa0dbp+0, 0x1.db72fc1f0eab4p-55, \
  0x1.8cf3216b5448cp+0, -0x1.5b6609cc5e7ffp-57, \
  0x1.8f1ae99157736p+0, 0x1.bf68359f35f44p-56, \
  0x1.9145b0b91ffc6p+0, -0x1.3091fa71e3d83p-54, \
  0x1.93737b0cdc5e5p+0, -0x1.da9b88b6c1e29p-58, \
  0x1.95a44cbc8520fp+0, -0x1.c23f97c90b959p-57, \
  0x1.97d829fde4e50p+0, -0x1.2434322f4f9aap-54, \
  0x1.9a0f170ca07bap+0, -0x1.5ca6cd7668e4bp-55, \
  0x1.9c49182a3f090p+0, 0x1.1affc2b91ce27p-56, \
  0x1.9e86319e32323p+0, 0x1.dd235e10a73bbp-57, \
  0x1.a0c667b5de565p+0, -0x1.7c50422622263p-55, \
  0x1.a309bec4a2d33p+0, 0x1.b1c86e3e231d5p-55, \
  0x1.a5503b23e255dp+0, -0x1.1bbd1d3bcbb15p-54, \
  0x1.a799e1330b358p+0, 0x1.0cc319cee31d2p-54, \
  0x1.a9e6b5579fdbfp+0, 0x1.469846e735ab3p-55, \
  0x1.ac36bbfd3f37ap+0, -0x1.2dfcd978e9db4p-55, \
  0x1.ae89f995ad3adp+0, 0x1.c1a7792cb3387p-55, \
  0x1.b0e07298db666p+0, -0x1.07b8f4ad1d9fap-54, \
  0x1.b33a2b84f15fbp+0, -0x1.5c3d956dcaebap-58, \
  0x1.b59728de5593ap+0, -0x1.0a40e3da6f640p-54, \
  0x1.b7f76f2fb5e47p+0, -0x1.8d6f438ad9334p-57, \
  0x1.ba5b030a1064ap+0, -0x1.1eee26b588a35p-54, \
  0x1.bcc1e904bc1d2p+0, 0x1.4ffd70a5fddcdp-56, \
  0x1.bf2c25bd71e09p+0, -0x1.1bdfbfa9298acp-54, \
  0x1.c199bdd85529cp+0, 0x1.36eae30af0cb3p-56, \
  0x1.c40ab5fffd07ap+0, 0x1.ee3325c9ffd94p-55, \
  0x1.c67f12e57d14bp+0, 0x1.4e08fd10959acp-55, \
  0x1.c8f6d9406e7b5p+0, 0x1.3cdaf384e1a67p-57, \
  0x1.cb720dcef9069p+0, 0x1.76b2c6c921968p-57, \
  0x1.cdf0b555dc3fap+0, -0x1.08a1883ccb5d2p-55, \
  0x1.d072d4a07897cp+0, -0x1.fad5d3ffffa6fp-55, \
  0x1.d2f87080d89f2p+0, -0x1.00dae3875a949p-54, \
  0x1.d5818dcfba487p+0, 0x1.4a385a63d07a7p-56, \
  0x1.d80e316c98398p+0, -0x1.2919e2040220fp-55, \
  0x1.da9e603db3285p+0, 0x1.e5a50d5c192acp-55, \
  0x1.dd321f301b460p+0, 0x1.43a59ac016b4bp-55, \
  0x1.dfc97337b9b5fp+0, -0x1.2d52107b43e1fp-55, \
  0x1.e264614f5a129p+0, -0x1.92ab93b470dc9p-55, \
  0x1.e502ee78b3ff6p+0, 0x1.4b604603a88d3p-56, \
  0x1.e7a51fbc74c83p+0, 0x1.3c5ec519d7271p-55, \
  0x1.ea4afa2a490dap+0, -0x1.ff7128fd391f0p-55, \
  0x1.ecf482d8e67f1p+0, -0x1.dae98e223747dp-55, \
  0x1.efa1bee615a27p+0, 0x1.ec3bc41aa2008p-55, \
  0x1.f252b376bba97p+0, 0x1.42b94c3a9eb32p-55, \
  0x1.f50765b6e4540p+0, 0x1.a64a931d185eep-55, \
  0x1.f7bfdad9cbe14p+0, -0x1.e37bae43be3edp-55, \
  0x1.fa7c1819e90d8p+0, 0x1.7893b4d91cd9dp-56, \
  0x1.fd3c22b8f71f1p+0, 0x1.305c14160cc89p-58 \
}
#define SG_LOG_OFF 0x3fe6000000000000ULL  /* bit pattern of 0.6875 */
#define SG_LOG_LN2_HI 0x1.62e42fefa3800p-1
#define SG_LOG_LN2_LO 0x1.ef35793c76730p-45
#define SG_LOG_C2 -0x1.0000000000000p-1  /* -1/2 */
#define SG_LOG_C3 0x1.5555555555555p-2  /* +1/3 */
#define SG_LOG_C4 -0x1.0000000000000p-2  /* -1/4 */
#define SG_LOG_C5 0x1.999999999999ap-3  /* +1/5 */
#define SG_LOG_C6 -0x1.5555555555555p-3  /* -1/6 */
#define SG_LOG_C7 0x1.2492492492492p-3  /* +1/7 */
#define SG_LOG_C8 -0x1.0000000000000p-3  /* -1/8 */
#define SG_LOG_C9 0x1.c71c71c71c71cp-4  /* +1/9 */
/* {c_j, hi(-log c_j), lo(-log c_j)} for the 128 subintervals of [0.6875, 1.375) */
#define SG_LOG_TAB_INIT { \
  0x1.734f0c541fe8dp+0, -0x1.7cc7f7db46a0ep-2, -0x1.e3c7fdc323c2dp-56, \
  0x1.713786d9c7c09p+0, -0x1.76feecb947176p-2, 0x1.398d9eb4ea363p-56, \
  0x1.6f26016f26017p+0, -0x1.713e33a46a17cp-2, 0x1.f6cf40b5c71a6p-57, \
  0x1.6d1a62681c861p+0, -0x1.6b85b4cffa3fdp-2, 0x1.1af2c8dafcb08p-57, \
  0x1.6b1490aa31a3dp+0, -0x1.65d558d4ce00bp-2, 0x1.4e05a4748480ap-56, \
  0x1.691473a88d0c0p+0, -0x1.602d08af091ecp-2, -0x1.a45db7cfd9230p-56, \
  0x1.6719f3601671ap+0, -0x1.5a8cadbbedfa1p-2, -0x1.64f5081307f22p-60, \
  0x1.6524f853b4aa3p+0, -0x1.54f431b7be1a8p-2, 0x1.0b3f6ef6ae452p-58, \
  0x1.63356b88ac0dep+0, -0x1.4f637ebba9810p-2, 0x1.68cb3124b9245p-56, \
  0x1.614b36831ae94p+0, -0x1.49da7f3bcc420p-2, 0x1.d964a168ccacbp-57, \
  0x1.5f66434292dfcp+0, -0x1.44591e0539f49p-2, -0x1.a76d6dc2782dap-59, \
  0x1.5d867c3ece2a5p+0, -0x1.3edf463c1683ep-2, 0x1.c852fe587def8p-57, \
  0x1.5babcc647fa91p+0, -0x1.396ce359bbf53p-2, 0x1.5c5663663d163p-59, \
  0x1.59d61f123ccaap+0, -0x1.3401e12aecba0p-2, -0x1.f95523adc5c9fp-57, \
  0x1.5805601580560p+0, -0x1.2e9e2bce12286p-2, 0x1.f3ed72e23e134p-57, \
  0x1.56397ba7c52e2p+0, -0x1.2941afb186b7cp-2, -0x1.6a4678ebaa300p-59, \
  0x1.54725e6bb82fep+0, -0x1.23ec5991eba49p-2, -0x1.76eba35bbf0dfp-61, \
  0x1.52aff56a8054bp+0, -0x1.1e9e1678899f5p-2, -0x1.64b0dd2687939p-58, \
  0x1.50f22e111c4c5p+0, -0x1.1956d3b9bc2f9p-2, -0x1.0e75a3542856fp-58, \
  0x1.4f38f62dd4c9bp+0, -0x1.14167ef367784p-2, -0x1.ef824daaf53e9p-56, \
  0x1.4d843bedc2c4cp+0, -0x1.0edd060b78082p-2, -0x1.2d4b610d7d4f5p-57, \
  0x1.4bd3edda68fe1p+0, -0x1.09aa572e6c6d4p-2, -0x1.f9e17343426a9p-56, \
  0x1.4a27fad76014ap+0, -0x1.047e60cde83b7p-2, -0x1.08869cbf9e344p-56, \
  0x1.4880522014880p+0, -0x1.feb2233ea07cbp-3, -0x1.8de00938b4c30p-61, \
  0x1.46dce34596066p+0, -0x1.f474b134df228p-3, 0x1.9f1df7b5daab7p-60, \
  0x1.453d9e2c776cap+0, -0x1.ea4449f04aaf5p-3, 0x1.f33919ab94074p-57, \
  0x1.43a2730abee4dp+0, -0x1.e020cc6235ab5p-3, 0x1.f0adb91423f18p-57, \
  0x1.420b5265e5951p+0, -0x1.d60a17f903514p-3, 0x1.50df841a71b7ap-57, \
  0x1.40782d10e6566p+0, -0x1.cc000c9db3c52p-3, -0x1.67a2a8500729ep-58, \
  0x1.3ee8f42a5af07p+0, -0x1.c2028ab17f9b5p-3, -0x1.c11aa3853a5f0p-57, \
  0x1.3d5d991aa75c6p+0, -0x1.b811730b823d4p-3, 0x1.d7c46328983c6p-58, \
  0x1.3bd60d9232955p+0, -0x1.ae2ca6f672bd8p-3, 0x1.a4a356155f779p-57, \
  0x1.3a524387ac822p+0, -0x1.a454082e6ab03p-3, 0x1.e0df823a3cb3dp-58, \
  0x1.38d22d366088ep+0, -0x1.9a8778debaa3ap-3, -0x1.28fbfb0e3f0fcp-58, \
  0x1.3755bd1c945eep+0, -0x1.90c6db9fcbcdbp-3, 0x1.357718d7ca4cfp-58, \
  0x1.35dce5f9f2af8p+0, -0x1.871213750e994p-3, 0x1.a97a0ca115d60p-57, \
  0x1.34679ace01346p+0, -0x1.7d6903caf5acdp-3, 0x1.0b17c301d6e14p-57, \
  0x1.32f5ced6a1dfap+0, -0x1.73cb9074fd14dp-3, 0x1.721a000b4cf01p-57, \
  0x1.3187758e9ebb6p+0, -0x1.6a399dabbd383p-3, -0x1.76332bd4b341fp-57, \
  0x1.301c82ac40260p+0, -0x1.60b3100b09474p-3, -0x1.526cee0fd7f4ap-57, \
  0x1.2eb4ea1fed14bp+0, -0x1.5737cc9018cddp-3, 0x1.00b28ef013c72p-57, \
  0x1.2d50a012d50a0p+0, -0x1.4dc7b897bc1c7p-3, -0x1.b60ae1ff0e82ep-59, \
  0x1.2bef98e5a3711p+0, -0x1.4462b9dc9b3dcp-3, 0x1.85388d830c709p-59, \
  0x1.2a91c92f3c105p+0, -0x1.3b08b6757f2a7p-3, -0x1.5e1ad9be0a4cdp-57, \
  0x1.293725bb804a5p+0, -0x1.31b994d3a4f86p-3, 0x1.1238b5efe0665p-57, \
  0x1.27dfa38a1ce4dp+0, -0x1.28753bc11aba2p-3, 0x1.7394d9fa33313p-57, \
  0x1.268b37cd60127p+0, -0x1.1f3b925f25d44p-3, -0x1.08b27be4e6b15p-57, \
  0x1.2539d7e9177b2p+0, -0x1.160c8024b27b0p-3, 0x1.355bfd870afebp-59, \
  0x1.23eb79717605bp+0, -0x1.0ce7ecdccc28bp-3, -0x1.1b57fea88da98p-59, \
  0x1.22a0122a0122ap+0, -0x1.03cdc0a51ec0dp-3, -0x1.19e2d3f8b7d10p-57, \
  0x1.21579804855e6p+0, -0x1.f57bc7d9005dbp-4, 0x1.d361574fb24e2p-58, \
  0x1.2012012012012p+0, -0x1.e3707ee30487bp-4, -0x1.9399d9aaf3b33p-59, \
  0x1.1ecf43c7fb84cp+0, -0x1.d179788219362p-4, 0x1.b12841044a96cp-58, \
  0x1.1d8f5672e4abdp+0, -0x1.bf968769fca18p-4, 0x1.06e4fb7af9c69p-58, \
  0x1.1c522fc1ce059p+0, -0x1.adc77ee5aea8ep-4, -0x1.d7d8f39bee658p-58, \
  0x1.1b17c67f2bae3p+0, -0x1.9c0c32d4d254dp-4, 0x1.627a0e199f569p-58, \
  0x1.19e0119e0119ep+0, -0x1.8a6477a91dc29p-4, 0x1.3d4190a482421p-58, \
  0x1.18ab083902bdbp+0, -0x1.78d02263d82d7p-4, -0x1.cbca5b4fdb87ep-58, \
  0x1.1778a191bd684p+0, -0x1.674f089365a78p-4, -0x1.ca64e9980e048p-59, \
  0x1.1648d50fc3201p+0, -0x1.55e10050e0382p-4, -0x1.9a0629e3973e4p-58, \
  0x1.151b9a3fdd5c9p+0, -0x1.4485e03dbdfb0p-4, -0x1.3ba349aadbc6dp-58, \
  0x1.13f0e8d344724p+0, -0x1.333d7f8183f4ap-4, 0x1.adaa06e211e9ep-59, \
  0x1.12c8b89edc0acp+0, -0x1.2207b5c7854a1p-4, -0x1.b3f0431efb154p-58, \
  0x1.11a3019a74826p+0, -0x1.10e45b3cae829p-4, -0x1.9b5ed72e6d974p-58, \
  0x1.107fbbe011080p+0, -0x1.ffa6911ab9309p-5, 0x1.cd9f1f95c2ef1p-59, \
  0x1.0f5edfab325a2p+0, -0x1.dda8adc67ee59p-5, 0x1.31936790bb3b2p-59, \
  0x1.0e40655826011p+0, -0x1.bbcebfc68f424p-5, 0x1.cd1862f854848p-59, \
  0x1.0d24456359e3ap+0, -0x1.9a187b573de81p-5, -0x1.b13b26f298a6ap-64, \
  0x1.0c0a7868b4171p+0, -0x1.788595a3577c8p-5, -0x1.2f7c4c5b3c8bdp-62, \
  0x1.0af2f722eecb5p+0, -0x1.5715c4c03cee1p-5, -0x1.5101dc4ebf91fp-59, \
  0x1.09ddba6af8360p+0, -0x1.35c8bfaa13069p-5, 0x1.50830a65543a8p-63, \
  0x1.08cabb37565e2p+0, -0x1.149e3e4005a8dp-5, 0x1.a9a4168fcebebp-60, \
  0x1.07b9f29b8eae2p+0, -0x1.e72bf2813ce6ap-6, 0x1.8a4bba6a354fap-60, \
  0x1.06ab59c7912fbp+0, -0x1.a55f548c5c427p-6, -0x1.f60d2fc36a0d9p-61, \
  0x1.059eea0727586p+0, -0x1.63d6178690bbep-6, 0x1.18ed4d357c9dcp-60, \
  0x1.04949cc1664c5p+0, -0x1.228fb1fea2e0ap-6, -0x1.3284991fe3d5cp-61, \
  0x1.038c6b78247fcp+0, -0x1.c317384c75f0dp-7, -0x1.806208c04c21fp-61, \
  0x1.02864fc7729e9p+0, -0x1.41929f968330cp-7, -0x1.3aae809b43dd0p-61, \
  0x1.0182436517a37p+0, -0x1.8121214586b02p-8, 0x1.c7d68c0d910f2p-62, \
  0x1.0000000000000p+0, 0x0.0p+0, 0x0.0p+0, \
  0x1.0000000000000p+0, 0x0.0p+0, 0x0.0p+0, \
  0x1.fa11caa01fa12p-1, 0x1.7dc475f810a69p-7, 0x1.74944bc161072p-61, \
  0x1.f6310aca0dbb5p-1, 0x1.3cea44346a584p-6, -0x1.865ad48159d00p-61, \
  0x1.f25f644230ab5p-1, 0x1.b9fc027af919ap-6, -0x1.90ae69229dc86p-60, \
  0x1.ee9c7f8458e02p-1, 0x1.1b0d98923d97fp-5, -0x1.74d7444dd6241p-59, \
  0x1.eae807aba01ebp-1, 0x1.58a5bafc8e4d3p-5, -0x1.cab8569c56e40p-64, \
  0x1.e741aa59750e4p-1, 0x1.95c830ec8e3f2p-5, 0x1.eb41d00a417e9p-60, \
  0x1.e3a9179dc1a73p-1, 0x1.d276b8adb0b56p-5, 0x1.078f14c95ff53p-59, \
  0x1.e01e01e01e01ep-1, 0x1.075983598e471p-4, 0x1.006d2999e22dcp-58, \
  0x1.dca01dca01dcap-1, 0x1.253f62f0a1417p-4, 0x1.1f6d34e01d981p-61, \
  0x1.d92f2231e7f8ap-1, 0x1.42edcbea646eep-4, -0x1.511583653349bp-58, \
  0x1.d5cac807572b2p-1, 0x1.60658a93750c4p-4, -0x1.f108b1d8436d3p-59, \
  0x1.d272ca3fc5b1ap-1, 0x1.7da766d7b12d0p-4, 0x1.a2240644d7da2p-59, \
  0x1.cf26e5c44bfc6p-1, 0x1.9ab42462033aep-4, -0x1.a099e1c184e8ep-59, \
  0x1.cbe6d9601cbe7p-1, 0x1.b78c82bb0eda0p-4, -0x1.3ef0e61f9b03cp-58, \
  0x1.c8b265afb8a42p-1, 0x1.d4313d66cb35dp-4, 0x1.b90dd951d90fap-58, \
  0x1.c5894d10d4986p-1, 0x1.f0a30c01162a4p-4, 0x1.8be64b8b7759bp-59, \
  0x1.c26b5392ea01cp-1, 0x1.0671512ca596fp-3, -0x1.2f39b81479b67p-58, \
  0x1.bf583ee868d8bp-1, 0x1.14785846742acp-3, 0x1.94409f1d3f83ap-60, \
  0x1.bc4fd65883e7bp-1, 0x1.2266f190a5acdp-3, -0x1.dab840e7f6177p-57, \
  0x1.b951e2b18ff23p-1, 0x1.303d718e47fd5p-3, -0x1.b5ae71f658247p-57, \
  0x1.b65e2e3beee05p-1, 0x1.3dfc2b0ecc62ap-3, 0x1.ba62b8c13f7f4p-57, \
  0x1.b37484ad806cep-1, 0x1.4ba36f39a55e5p-3, -0x1.f767e433c98aap-57, \
  0x1.b094b31d922a4p-1, 0x1.59338d9982085p-3, 0x1.8d16eaaba9419p-57, \
  0x1.adbe87f94905ep-1, 0x1.66acd4272ad51p-3, -0x1.9201c9c3d5165p-59, \
  0x1.aaf1d2f87ebfdp-1, 0x1.740f8f54037a3p-3, 0x1.6d9bf9d57b326p-58, \
  0x1.a82e65130e159p-1, 0x1.815c0a14357e9p-3, 0x1.141b7f8c5fa9ep-58, \
  0x1.a574107688a4ap-1, 0x1.8e928de886d41p-3, 0x1.2589eb96a6240p-59, \
  0x1.a2c2a87c51ca0p-1, 0x1.9bb362e7dfb85p-3, -0x1.51439c1ff83e7p-58, \
  0x1.a01a01a01a01ap-1, 0x1.a8becfc882f19p-3, -0x1.a8c37918c39ebp-58, \
  0x1.9d79f176b682dp-1, 0x1.b5b519e8fb5a6p-3, -0x1.d5d8023e61e5fp-57, \
  0x1.9ae24ea5510dap-1, 0x1.c2968558c18c2p-3, 0x1.6108e3ae024acp-60, \
  0x1.9852f0d8ec0ffp-1, 0x1.cf6354e09c5ddp-3, 0x1.339a07d55b696p-57, \
  0x1.95cbb0be377aep-1, 0x1.dc1bca0abec7bp-3, 0x1.c698a33316dfbp-58, \
  0x1.934c67f9b2ce6p-1, 0x1.e8c0252aa5a60p-3, -0x1.dc074737f9135p-60, \
  0x1.90d4f120190d5p-1, 0x1.f550a564b7b37p-3, -0x1.13a09202fe73dp-57, \
  0x1.8e6527af1373fp-1, 0x1.00e6c45ad501dp-2, -0x1.3b9568ff6feadp-57, \
  0x1.8bfce8062ff3ap-1, 0x1.071b85fcd590dp-2, 0x1.08b83fcbdef40p-57, \
  0x1.899c0f601899cp-1, 0x1.0d46b579ab74bp-2, 0x1.21f640e1e5ec9p-56, \
  0x1.87427bcc092b9p-1, 0x1.136870293a8b0p-2, 0x1.86cc531dba494p-57, \
  0x1.84f00c2780614p-1, 0x1.1980d2dd4236fp-2, -0x1.02c2e4f1b2eb9p-56, \
  0x1.82a4a0182a4a0p-1, 0x1.1f8ff9e48a2f3p-2, -0x1.93fbf3418960dp-57, \
  0x1.8060180601806p-1, 0x1.2596010df763ap-2, -0x1.9eed8ae0ebd3cp-59, \
  0x1.7e225515a4f1dp-1, 0x1.2b9303ab89d25p-2, -0x1.85ad7f614ab51p-58, \
  0x1.7beb3922e017cp-1, 0x1.31871c9544185p-2, -0x1.ea3598981366fp-57, \
  0x1.79baa6bb6398bp-1, 0x1.3772662bfd85cp-2, 0x1.02a7589fba088p-57, \
  0x1.77908119ac60dp-1, 0x1.3d54fa5c1f710p-2, 0x1.53668e578d9cdp-58, \
  0x1.756cac201756dp-1, 0x1.432ef2a04e813p-2, -0x1.83262e2b59206p-57 \
}
/* correctly rounded exp/log (sg_crmath.h) */
#define SG_CR_EXP_XMAX 0x1.62e42fefa39efp+9  /* largest x with RN(exp(x)) finite */
#define SG_CR_EXP_XMIN -0x1.74910d52d3051p+9  /* smallest x with RN(exp(x)) > 0 */
#define SG_CR_EXP_C1 0x1.62e42fef80000p-8
#define SG_CR_EXP_C2 0x1.1cf79abc80000p-43
#define SG_CR_EXP_C3 0x1.e3b39803f2f6bp-79
#define SG_CR_EXP_F2_HI 0x1.0000000000000p-1
#define SG_CR_EXP_F2_LO 0x0.0p+0
#define SG_CR_EXP_F3_HI 0x1.5555555555555p-3
#define SG_CR_EXP_F3_LO 0x1.5555555555555p-57
#define SG_CR_EXP_F4_HI 0x1.5555555555555p-5
#define SG_CR_EXP_F4_LO 0x1.5555555555555p-59
#define SG_CR_EXP_F5_HI 0x1.1111111111111p-7
#define SG_CR_EXP_F5_LO 0x1.1111111111111p-63
#define SG_CR_EXP_F6 0x1.6c16c16c16c17p-10
#define SG_CR_EXP_F7 0x1.a01a01a01a01ap-13
#define SG_CR_EXP_F8 0x1.a01a01a01a01ap-16
#define SG_CR_EXP_F9 0x1.71de3a556c734p-19
#define SG_CR_EXP_F10 0x1.27e4fb7789f5cp-22
#define SG_CR_EXP_F11 0x1.ae64567f544e4p-26
#define SG_CR_LOG_LN2_LO2 0x1.f97b57a079a19p-103
#define SG_CR_LOG_G2_HI -0x1.0000000000000p-1
#define SG_CR_LOG_G2_LO 0x0.0p+0
#define SG_CR_LOG_G2 -0x1.0000000000000p-1
#define SG_CR_LOG_G3_HI 0x1.5555555555555p-2
#define SG_CR_LOG_G3_LO 0x1.5555555555555p-56
#define SG_CR_LOG_G3 0x1.5555555555555p-2
#define SG_CR_LOG_G4_HI -0x1.0000000000000p-2
#define SG_CR_LOG_G4_LO 0x0.0p+0
#define SG_CR_LOG_G4 -0x1.0000000000000p-2
#define SG_CR_LOG_G5_HI 0x1.999999999999ap-3
#define SG_CR_LOG_G5_LO -0x1.999999999999ap-57
#define SG_CR_LOG_G5 0x1.999999999999ap-3
#define SG_CR_LOG_G6_HI -0x1.5555555555555p-3
#define SG_CR_LOG_G6_LO -0x1.5555555555555p-57
#define SG_CR_LOG_G6 -0x1.5555555555555p-3
#define SG_CR_LOG_G7_HI 0x1.2492492492492p-3
#define SG_CR_LOG_G7_LO 0x1.2492492492492p-57
#define SG_CR_LOG_G7 0x1.2492492492492p-3
#define SG_CR_LOG_G8_HI -0x1.0000000000000p-3
#define SG_CR_LOG_G8_LO 0x0.0p+0
#define SG_CR_LOG_G8 -0x1.0000000000000p-3
#define SG_CR_LOG_G9_HI 0x1.c71c71c71c71cp-4
#define SG_CR_LOG_G9_LO 0x1.c71c71c71c71cp-58
#define SG_CR_LOG_G9 0x1.c71c71c71c71cp-4
#define SG_CR_LOG_G10 -0x1.999999999999ap-4
#define SG_CR_LOG_G11 0x1.745d1745d1746p-4
#define SG_CR_LOG_G12 -0x1.5555555555555p-4
#define SG_CR_LOG_G13 0x1.3b13b13b13b14p-4
#define SG_CR_LOG_G14 -0x1.2492492492492p-4
#define SG_CR_LOG_G15 0x1.1111111111111p-4
#define SG_CR_LOG_G16 -0x1.0000000000000p-4
#define SG_CR_LOG_G17 0x1.e1e1e1e1e1e1ep-5
